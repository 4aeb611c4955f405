"""Pins the CPU oracle to answers computed outside this repository.

- GF(2^128): the NIST CAVP GCM vectors the reference ships
  (crates/field/tests/ghash_vectors.rs), via tests/golden/ghash_nist.json.
- SHA-256 / SHA3-256 (Keccak-f): Python hashlib; FIPS 180-4 "abc".
- BLAKE3: the published digests of "" and "abc"; hash and derive-key mode
  over 0 bytes to 100 chunks from the BLAKE3 team's implementation, via
  tests/golden/blake3_vectors.json.
- The narg layout of the reference's golden transcript (crates/transcript/tests/golden.rs:14).
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import ffi as of

HERE = os.path.dirname(os.path.abspath(__file__))


def _rb(b):
    return bytes(int(f"{x:08b}"[::-1], 2) for x in b)


def _from_nist(b):
    b = _rb(b)
    return np.array([int.from_bytes(b[:8], "little"), int.from_bytes(b[8:], "little")], dtype=np.uint64)


def _to_nist(f):
    return _rb(int(f[0]).to_bytes(8, "little") + int(f[1]).to_bytes(8, "little"))


@pytest.mark.parametrize("mode", [0, 1])
def test_ghash_matches_nist_gcm_vectors(mode):
    of.lib().o_set_clmul_mode(mode)
    fx = json.load(open(os.path.join(HERE, "golden", "ghash_nist.json")))
    assert len(fx["cases"]) == 525
    for i, c in enumerate(fx["cases"]):
        h = _from_nist(bytes.fromhex(c["h"]))
        x = np.zeros(2, dtype=np.uint64)

        def absorb(data, x):
            for k in range(0, len(data), 16):
                y = _from_nist(data[k:k + 16].ljust(16, b"\0"))
                x = of.gf_mul(x ^ y, h)
            return x

        aad, ct = bytes.fromhex(c["aad"]), bytes.fromhex(c["ct"])
        x = absorb(aad, x)
        x = absorb(ct, x)
        lengths = (len(aad) * 8).to_bytes(8, "big") + (len(ct) * 8).to_bytes(8, "big")
        x = of.gf_mul(x ^ _from_nist(lengths), h)
        want = c["ghash_prefix"]
        assert _to_nist(x)[: len(want) // 2].hex() == want, f"case {i}"
    of.lib().o_set_clmul_mode(0)


def test_inverse_and_reduction_boundary():
    rng = np.random.default_rng(7)
    one = np.array([1, 0], dtype=np.uint64)
    for _ in range(20):
        a = rng.integers(0, 2**64, size=2, dtype=np.uint64)
        r = of.lib().o_gf_inv(of.F128(int(a[0]), int(a[1])))
        assert np.array_equal(of.gf_mul(a, np.array([r.lo, r.hi], dtype=np.uint64)), one)
    # X^127 * X = X^128 = X^7 + X^2 + X + 1 (crates/field/src/gf128.rs:453-462)
    x127 = np.array([0, 1 << 63], dtype=np.uint64)
    x = np.array([2, 0], dtype=np.uint64)
    assert np.array_equal(of.gf_mul(x127, x), np.array([0x87, 0], dtype=np.uint64))


@pytest.mark.parametrize("msg", [b"", b"abc", b"a" * 55, b"a" * 56, b"a" * 64, bytes(range(256)) * 5])
def test_sha256_and_sha3_match_hashlib(msg):
    buf = ctypes.create_string_buffer(32)
    of.lib().o_sha256(msg, len(msg), buf)
    assert buf.raw == hashlib.sha256(msg).digest()
    of.lib().o_sha3_256(msg, len(msg), buf)
    assert buf.raw == hashlib.sha3_256(msg).digest()


def test_sha256_fips_abc():
    buf = ctypes.create_string_buffer(32)
    of.lib().o_sha256(b"abc", 3, buf)
    # FIPS 180-4 "abc" digest (crates/circuit/src/sha256.rs:34-37)
    assert buf.raw.hex() == "ba7816bf8f01cfea414140de5dae2223b00361a396177a9cb410ff61f20015ad"


def test_blake3_published_digests():
    buf = ctypes.create_string_buffer(32)
    of.lib().o_blake3(b"", 0, buf)
    assert buf.raw.hex() == "af1349b9f5f9a1a6a0404dea36dcc9499bcb25c9adc112b7cc9a93cae41f3262"
    of.lib().o_blake3(b"abc", 3, buf)
    assert buf.raw.hex() == "6437b3ac38465133ffb63b75273a8db548c558465d79db03fd359c6cd5bd9d85"


def _blake3_vectors():
    import json
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "blake3_vectors.json")
    return json.load(open(path))


def _blake3_input(n):
    return bytes(i % 251 for i in range(n))


def test_blake3_tree_mode_known_answers():
    """Hash mode from 0 bytes to 100 chunks: every chunk boundary and parent
    merge of the chunk tree (fixture: tests/golden/make_blake3_fixture.py)."""
    vec = _blake3_vectors()
    buf = ctypes.create_string_buffer(32)
    for case in vec["cases"]:
        x = _blake3_input(case["len"])
        of.lib().o_blake3(x, len(x), buf)
        assert buf.raw.hex() == case["hash"], case["len"]


def test_blake3_derive_key_known_answers():
    """Derive-key mode (the weight digest's, crates/pcs/src/opening.rs:354-365)
    for the path's context and the test-vector context, fed whole and in
    uneven pieces."""
    vec = _blake3_vectors()
    buf = ctypes.create_string_buffer(32)
    for case in vec["cases"]:
        x = _blake3_input(case["len"])
        for ctx in vec["contexts"]:
            for piece in (0, 1, 63, 1000, 4096):
                if piece == 1 and case["len"] > 8192:
                    continue
                of.lib().o_blake3_derive_key(ctx.encode(), x, len(x), piece, buf)
                assert buf.raw.hex() == case["derive_key"][ctx], (case["len"], ctx, piece)


GOLDEN_C1 = "1d1bcda36aa1541c3752f7b23fedef81"
GOLDEN_C2 = "e80729d4aa76e8e4d28dd085143eb3d5"


def _golden_events(t):
    """The event sequence of crates/transcript/tests/golden.rs:22-30 (the hint
    goes to the hint stream, not the sponge); returns (c1, c2) as bytes."""
    msg = (0x0123456789ABCDEF).to_bytes(8, "little") + (0xFEDCBA9876543210).to_bytes(8, "little")
    t.prover_message(msg)
    c1 = t.verifier_message_f128()
    t.prover_message((12345).to_bytes(16, "little"))
    c2 = t.verifier_message_f128()
    as_bytes = lambda c: int(c[0]).to_bytes(8, "little") + int(c[1]).to_bytes(8, "little")
    return as_bytes(c1), as_bytes(c2)


def test_golden_transcript_narg_layout():
    """crates/transcript/tests/golden.rs:7-38: the narg string is the F128 message
    (16 B LE, lo then hi) then the Fq message (16 B LE canonical); the hint stays out."""
    t = of.Transcript(b"golden-session", b"golden-instance")
    _golden_events(t)
    assert t.narg().hex() == "efcdab89674523011032547698badcfe39300000000000000000000000000000"


@pytest.mark.xfail(strict=True, reason=(
    "golden challenges NOT reproduced: spongefish 0.7.4 (its DomainSeparator, protocol_id, "
    "session/instance absorption and duplex rules) is not in the reference tree, and no "
    "candidate framing searched reproduces C1"))
def test_golden_transcript_challenges():
    """crates/transcript/tests/golden.rs:16-17 pins the two squeezed challenges.
    The sponge here is a Keccak-f[1600] duplex (rate 136) framed from the
    reference's own description; this test states the pin and records that it
    is not met."""
    c1, c2 = _golden_events(of.Transcript(b"golden-session", b"golden-instance"))
    assert c1.hex() == GOLDEN_C1
    assert c2.hex() == GOLDEN_C2

def test_product_host_blake3_known_answers():
    """The product library's host BLAKE3 (grinding, Merkle checks, the weight
    digest's root) against the same known answers, both modes."""
    from bitz_b200 import _lib
    lib = _lib.load()
    vec = _blake3_vectors()
    out = (ctypes.c_uint8 * 32)()
    for case in vec["cases"]:
        x = _blake3_input(case["len"])
        assert lib.bitz_blake3(None, x, len(x), out) == 0
        assert bytes(out).hex() == case["hash"], case["len"]
        for ctx in vec["contexts"]:
            assert lib.bitz_blake3(ctx.encode(), x, len(x), out) == 0
            assert bytes(out).hex() == case["derive_key"][ctx], (case["len"], ctx)
