"""The product verifier (bitz_verify, CircuitProofSystem::verify of
tooling/cli/src/end_to_end.rs:339-377, run by this library with its bulk steps
on the device): it accepts GPU proofs of every workload, agrees with the
oracle's restated verifier, and rejects every tampered byte range,
truncation, extension, a proof checked against a different statement or
security level, and swapped proofs."""
import struct

import pytest

import bitz_b200 as bz
from bitz_b200 import statements as ci
from oracle import ffi as of

pytestmark = pytest.mark.gpu

CASES = [("sha256-compression", 1, 100), ("sha256-compression", 1, 128),
         ("sha256-block-aligned", 0, 100), ("sha256-chain", 2, 100),
         ("sha256-block-aligned", 1, 128)]
FULL = [("sha256-chain", 64, 1, 100), ("sha256-block-aligned", 32, 3, 100),
        ("sha256-2kb", 32, 4, 128), ("sha256-chain", 1024, 2, 128)]


def statement(kind, blocks):
    st = ci.random_state(2) if kind == "sha256-compression" else None
    inp, out, _ = ci.instance(kind, blocks, 11 + blocks, st)
    return inp, out


@pytest.fixture(scope="module")
def proofs():
    out = {}
    for kind, blocks, sec in CASES:
        inp, outp = statement(kind, blocks)
        ps = bz.CircuitProofSystem(kind, inp, outp, sec)
        out[(kind, blocks, sec)] = (ps, inp, outp, ps.prove()[0])
    return out


def rejects(ps, proof):
    with pytest.raises(bz.BitzError) as e:
        ps.verify(proof)
    assert e.value.code in ("VerifyError", "MalformedProof"), str(e.value)
    return e.value


@pytest.mark.parametrize("case", CASES)
def test_accepts_gpu_proofs(proofs, case):
    ps, inp, outp, proof = proofs[case]
    ps.verify(proof)
    of.lib().o_set_clmul_mode(1)
    assert of.verify(ci.KINDS[case[0]], inp, outp, case[2], proof) == 0


@pytest.mark.parametrize("kind,blocks,seed,security", FULL)
def test_accepts_full_size_proofs(kind, blocks, seed, security):
    inp, out, _ = ci.instance(kind, blocks, seed)
    ps = bz.CircuitProofSystem(kind, inp, out, security)
    proof, _ = ps.prove()
    ps.verify(proof)
    bad = bytearray(proof)
    bad[len(bad) // 2] ^= 0x10
    rejects(ps, bytes(bad))


def sections(proof):
    i = proof.index(b"bitzPCS\x00")
    narg_len, hints_len = struct.unpack_from("<QQ", proof, i + 16)
    start = i + 32
    return i, start, start + narg_len, start + narg_len + hints_len


def test_rejects_every_tampered_region(proofs):
    ps, inp, outp, proof = proofs[("sha256-compression", 1, 100)]
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
            rejects(ps, bytes(bad))
    ps.verify(proof)  # the lane is still usable after all the rejections


def test_rejects_truncated_and_extended(proofs):
    ps, _, _, proof = proofs[("sha256-chain", 2, 100)]
    for bad in (proof[:-1], proof + b"\x00", proof[:100], b"", proof[:40]):
        rejects(ps, bad)
    assert rejects(ps, proof[:-1]).code == "MalformedProof"


def test_rejects_another_statement(proofs):
    _, inp, outp, proof = proofs[("sha256-chain", 2, 100)]
    wrong_out = outp.copy()
    wrong_out[17] ^= 1
    rejects(bz.CircuitProofSystem("sha256-chain", inp, wrong_out, 100), proof)
    wrong_in = inp.copy()
    wrong_in[3] ^= 1
    rejects(bz.CircuitProofSystem("sha256-chain", wrong_in, outp, 100), proof)


def test_rejects_the_other_security_level(proofs):
    _, inp, outp, proof = proofs[("sha256-compression", 1, 100)]
    rejects(bz.CircuitProofSystem("sha256-compression", inp, outp, 128), proof)
    _, inp, outp, proof = proofs[("sha256-compression", 1, 128)]
    rejects(bz.CircuitProofSystem("sha256-compression", inp, outp, 100), proof)


def test_rejects_swapped_proofs(proofs):
    a = proofs[("sha256-compression", 1, 100)]
    b = proofs[("sha256-chain", 2, 100)]
    rejects(a[0], b[3])
    rejects(b[0], a[3])
