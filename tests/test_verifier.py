"""The restated verifier (oracle/prover.cpp, CircuitProofSystem::verify of
tooling/cli/src/end_to_end.rs:339-377): it accepts the prover's proofs and
rejects every tampered byte range, truncation, extension, and a proof checked
against a different statement or security level."""
import struct

import numpy as np
import pytest

from bitz_b200 import statements as ci
from oracle import ffi as of


@pytest.fixture(autouse=True)
def fast_oracle():
    of.lib().o_set_clmul_mode(1)
    yield
    of.lib().o_set_clmul_mode(0)


CASES = [("sha256-compression", 1, 100), ("sha256-compression", 1, 128),
         ("sha256-block-aligned", 0, 100), ("sha256-chain", 2, 100), ("sha256-block-aligned", 1, 128)]


def statement(kind, blocks):
    st = ci.random_state(2) if kind == "sha256-compression" else None
    inp, out, _ = ci.instance(kind, blocks, 11 + blocks, st)
    return inp, out


@pytest.fixture(scope="module")
def proofs():
    of.lib().o_set_clmul_mode(1)
    out = {}
    for kind, blocks, sec in CASES:
        inp, outp = statement(kind, blocks)
        rc, proof, _ = of.prove(ci.KINDS[kind], inp, outp, sec)
        assert rc == 0
        out[(kind, blocks, sec)] = (inp, outp, proof)
    return out


def sections(proof):
    """Byte ranges of the container: (narg start, narg end, hints end)."""
    i = proof.index(b"bitzPCS\x00")
    narg_len, hints_len = struct.unpack_from("<QQ", proof, i + 16)
    start = i + 32
    return i, start, start + narg_len, start + narg_len + hints_len


@pytest.mark.parametrize("case", CASES)
def test_accepts_honest_proofs(proofs, case):
    inp, outp, proof = proofs[case]
    assert of.verify(ci.KINDS[case[0]], inp, outp, case[2], proof) == 0


def test_rejects_every_tampered_region(proofs):
    case = ("sha256-compression", 1, 100)
    inp, outp, proof = proofs[case]
    box, n0, n1, h1 = sections(proof)
    assert h1 == len(proof)
    spots = {
        "root": 3, "outer sumcheck": 40, "abc claims": box - 16 * 3 * 14 - 40,
        "inner sumcheck": box - 20, "container header": box + 9,
        "ood value": n0 + 3, "folds": n0 + 16 + 100, "mid narg": (n0 + n1) // 2,
        "late narg": n1 - 40, "last narg byte": n1 - 1, "hint length": n1 + 1,
        "first opened row": n1 + 4 + 8 + 5, "mid hints": (n1 + h1) // 2, "last byte": h1 - 1,
    }
    for name, at in spots.items():
        for bit in (0, 7):
            bad = bytearray(proof)
            bad[at] ^= 1 << bit
            assert of.verify(ci.KINDS[case[0]], inp, outp, case[2], bytes(bad)) != 0, (name, bit)


def test_rejects_truncated_and_extended(proofs):
    case = ("sha256-chain", 2, 100)
    inp, outp, proof = proofs[case]
    k = ci.KINDS[case[0]]
    assert of.verify(k, inp, outp, 100, proof[:-1]) != 0
    assert of.verify(k, inp, outp, 100, proof + b"\x00") != 0
    assert of.verify(k, inp, outp, 100, proof[:100]) != 0
    assert of.verify(k, inp, outp, 100, b"") != 0


def test_rejects_another_statement(proofs):
    case = ("sha256-chain", 2, 100)
    inp, outp, proof = proofs[case]
    k = ci.KINDS[case[0]]
    wrong_out = outp.copy()
    wrong_out[17] ^= 1
    assert of.verify(k, inp, wrong_out, 100, proof) != 0
    wrong_in = inp.copy()
    wrong_in[3] ^= 1
    assert of.verify(k, wrong_in, outp, 100, proof) != 0


def test_rejects_the_other_security_level(proofs):
    case = ("sha256-compression", 1, 100)
    inp, outp, proof = proofs[case]
    assert of.verify(ci.KINDS[case[0]], inp, outp, 128, proof) != 0
    case = ("sha256-compression", 1, 128)
    inp, outp, proof = proofs[case]
    assert of.verify(ci.KINDS[case[0]], inp, outp, 100, proof) != 0


def test_rejects_swapped_proofs(proofs):
    a = proofs[("sha256-compression", 1, 100)]
    b = proofs[("sha256-chain", 2, 100)]
    assert of.verify(ci.KINDS["sha256-compression"], a[0], a[1], 100, b[2]) != 0
    assert of.verify(ci.KINDS["sha256-chain"], b[0], b[1], 100, a[2]) != 0
