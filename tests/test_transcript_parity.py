"""The product's host transcript (libbitz_b200.so) against the oracle's, byte for byte.

Runs on CPU: the transcript is host code (Fiat-Shamir stays on the host)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import bitz_b200 as bz
from oracle import ffi as of


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_event_sequences_agree(seed):
    rng = np.random.default_rng(seed)
    p = bz.build_prover(b"bitz/circuit-e2e/v2", b"sha256-chain")
    o = of.Transcript(b"bitz/circuit-e2e/v2", b"sha256-chain")
    for _ in range(60):
        kind = rng.integers(0, 4)
        if kind == 0:
            msg = rng.bytes(int(rng.integers(0, 400)))
            p.public_message(msg)
            o.public_message(msg)
        elif kind == 1:
            msg = rng.bytes(int(rng.integers(1, 300)))
            p.prover_message(msg)
            o.prover_message(msg)
        elif kind == 2:
            assert np.array_equal(p.verifier_message_f128(), o.verifier_message_f128())
        else:
            bits = int(rng.integers(0, 9))
            p.grind(b"gkr/cubic/v1", bits)
            o.grind(b"gkr/cubic/v1", bits)
    assert p.narg() == o.narg()
    assert np.array_equal(p.verifier_message_f128(), o.verifier_message_f128())


def test_grinding_nonces_agree_at_every_difficulty():
    # The library searches sixteen nonces per step; the oracle tries them one
    # at a time. Both must send the smallest passing nonce, wherever it falls
    # within a step of sixteen (difficulties 1-20, several seeds each up to 12;
    # the higher ones reach nonces whose bytes 1 and 2 are set).
    for bits in range(1, 21):
        for s in range(4 if bits <= 12 else 1):
            session = b"grind-%d-%d" % (bits, s)
            p = bz.build_prover(session, b"pow")
            o = of.Transcript(session, b"pow")
            p.grind(b"bitz/pcs/sumcheck/v1", bits)
            o.grind(b"bitz/pcs/sumcheck/v1", bits)
            assert p.narg() == o.narg(), (bits, s)
            assert np.array_equal(p.verifier_message_f128(), o.verifier_message_f128())


def test_prime_sampling_agrees_and_is_prime():
    import ctypes
    p = bz.build_prover(b"s", b"prime")
    o = of.Transcript(b"s", b"prime")
    for bits in (20, 64, 121):
        q = p.squeeze_prime(bits)
        buf = ctypes.create_string_buffer(16)
        of.lib().o_ts_prime_le(ctypes.c_void_p(o.h), bits, buf)
        assert q == int.from_bytes(buf.raw, "little")
        assert q.bit_length() == bits and q % 2 == 1
        # Fermat check with Python big integers
        for base in (2, 3, 5, 7, 11):
            assert pow(base, q - 1, q) == 1


def _oracle_prime(o, bits):
    import ctypes
    buf = ctypes.create_string_buffer(16)
    of.lib().o_ts_prime_le(ctypes.c_void_p(o.h), bits, buf)
    return int.from_bytes(buf.raw, "little")


# Sessions (empty instance) in which a composite candidate passes its first
# strong round and fails a later one: the library runs the remaining rounds
# together, so it must put the sponge back and redraw exactly the bases the
# oracle's round-at-a-time loop draws.
@pytest.mark.parametrize("session,bits", [
    (b"rb-14-2554", 14), (b"rb-14-3623", 14), (b"rb-16-261", 16),
    (b"rb-16-518", 16), (b"rb-18-331", 18), (b"rb-18-902", 18)])
def test_prime_sampling_after_a_round_zero_liar(session, bits):
    p = bz.build_prover(session, b"")
    o = of.Transcript(session, b"")
    assert p.squeeze_prime(bits) == _oracle_prime(o, bits)
    assert np.array_equal(p.verifier_message_f128(), o.verifier_message_f128())


def test_prime_sampling_agrees_over_many_sessions():
    for i in range(150):
        session = b"many-%d" % i
        bits = (121, 64, 40)[i % 3]
        p = bz.build_prover(session, b"prime")
        o = of.Transcript(session, b"prime")
        assert p.squeeze_prime(bits) == _oracle_prime(o, bits), (i, bits)
        assert np.array_equal(p.verifier_message_f128(), o.verifier_message_f128())


def test_hints_bypass_the_sponge():
    a = bz.build_prover(b"s", b"i")
    b = bz.build_prover(b"s", b"i")
    a.hint(b"\xaa" * 5)
    assert np.array_equal(a.verifier_message_f128(), b.verifier_message_f128())
    assert a.hints() == b"\xaa" * 5 and a.narg() == b""


@pytest.mark.skipif(os.environ.get("BITZ_HOST_SIMD") == "0", reason="already the scalar paths")
def test_scalar_host_paths_agree_too():
    # BITZ_HOST_SIMD=0 selects the one-nonce-at-a-time grind, the
    # thread-pool strong rounds and the general-register Keccak permutation
    # (the paths of hosts without AVX-512); the event-sequence, grinding and
    # prime tests above rerun on them in a fresh process.
    env = dict(os.environ, BITZ_HOST_SIMD="0")
    r = subprocess.run(
        [sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", __file__,
         "-k", "event_sequence or grinding or prime"],
        env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def test_golden_event_sequence_agrees():
    """The reference's golden event sequence (crates/transcript/tests/golden.rs:22-30)
    gives the same narg, hints and challenges through the product's transcript
    as through the oracle's (whose golden-challenge pin is recorded as not met
    in test_oracle_pins.py)."""
    msg = (0x0123456789ABCDEF).to_bytes(8, "little") + (0xFEDCBA9876543210).to_bytes(8, "little")
    p = bz.build_prover(b"golden-session", b"golden-instance")
    o = of.Transcript(b"golden-session", b"golden-instance")
    for t in (p, o):
        t.prover_message(msg)
    assert np.array_equal(p.verifier_message_f128(), o.verifier_message_f128())
    p.hint(b"\xaa" * 5)
    for t in (p, o):
        t.prover_message((12345).to_bytes(16, "little"))
    assert np.array_equal(p.verifier_message_f128(), o.verifier_message_f128())
    assert p.narg() == o.narg()
    assert p.narg().hex() == "efcdab89674523011032547698badcfe39300000000000000000000000000000"
    assert p.hints().hex() == "aaaaaaaaaa"
