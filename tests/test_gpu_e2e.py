"""End-to-end parity: the GPU prover's proof bytes against the CPU oracle's.

Every Fiat-Shamir challenge depends on every earlier message, so equal proof
bytes mean every stage (witness, commitment, Spartan, fold, GKR, M^T,
post-GKR, ring switch, Ligerito) produced identical values."""
import numpy as np
import pytest

import bitz_b200 as bz
from bitz_b200 import statements as ci
from oracle import ffi as of

pytestmark = pytest.mark.gpu

CASES = [("sha256-compression", 1, 100), ("sha256-block-aligned", 0, 128),
         ("sha256-chain", 2, 100), ("sha256-block-aligned", 1, 100), ("sha256-chain", 3, 128)]


@pytest.fixture(autouse=True)
def fast_oracle():
    of.lib().o_set_clmul_mode(1)
    yield
    of.lib().o_set_clmul_mode(0)


def first_difference(a: bytes, b: bytes):
    n = min(len(a), len(b))
    for i in range(n):
        if a[i] != b[i]:
            return i
    return None if len(a) == len(b) else n


@pytest.mark.parametrize("kind,blocks,security", CASES)
def test_proof_bytes_match_oracle(kind, blocks, security):
    st = ci.random_state(2) if kind == "sha256-compression" else None
    inp, out, _ = ci.instance(kind, blocks, 11 + blocks, st)
    rc, oproof, _ = of.prove(ci.KINDS[kind], inp, out, security)
    assert rc == 0
    ps = bz.CircuitProofSystem(kind, inp, out, security)
    gproof, times = ps.prove()
    assert first_difference(gproof, oproof) is None, (len(gproof), len(oproof))


# Every single-proof workload at its full size: the benchmark statement
# (sha256-chain n=64, seed 1), the large one (n=1024, seed 2, 128-bit
# profile: unique decoding, four PCS levels, m_f = 23), block-aligned k=32
# and the 2 KiB message.
FULL_SIZE = [("sha256-chain", 64, 1, 100), ("sha256-block-aligned", 32, 3, 100),
             ("sha256-2kb", 32, 4, 128), ("sha256-chain", 1024, 2, 128)]


@pytest.mark.parametrize("kind,blocks,seed,security", FULL_SIZE)
def test_full_size_proof_bytes_match_oracle(kind, blocks, seed, security):
    inp, out, _ = ci.instance(kind, blocks, seed)
    rc, oproof, _ = of.prove(ci.KINDS[kind], inp, out, security)
    assert rc == 0
    gproof, _ = bz.CircuitProofSystem(kind, inp, out, security).prove()
    assert first_difference(gproof, oproof) is None, (len(gproof), len(oproof),
                                                      first_difference(gproof, oproof))


def test_batch_mix_proofs_match_oracle():
    """Eight statements of the batched workload (block-aligned, uneven k),
    proved together on four lanes, each equal to the oracle's proof."""
    mix = ci.batch_mix(3, 256, 32)[:8]
    systems = [bz.CircuitProofSystem(kind, inp, out, 100) for kind, inp, out in mix]
    proofs, _ = bz.batch_prove(systems, 4)
    for (kind, inp, out), proof in zip(mix, proofs):
        rc, oproof, _ = of.prove(ci.KINDS[kind], inp, out, 100)
        assert rc == 0
        assert first_difference(proof, oproof) is None, (kind, len(inp) // 512)


@pytest.mark.parametrize("blocks,seed", [(2, 3), (64, 1)])
def test_witness_matches_oracle(blocks, seed):
    inp, out, _ = ci.instance("sha256-chain", blocks, seed)
    oc = of.Circuit(1, inp, out)
    ps = bz.CircuitProofSystem("sha256-chain", inp, out, 100)
    ps.prove()
    s = ps.stats()
    f, h, prod = ps.witness_parts((s["padded_committed_bits"]) // 32, (1 << (s["claim_log_cols"] + 7)) // 32,
                            s["constraints"])
    fb = np.unpackbits(f.view(np.uint8), bitorder="little")
    hb = np.unpackbits(h.view(np.uint8), bitorder="little")
    assert np.array_equal(fb[: oc.f_len], oc.f()) and not fb[oc.f_len:].any()
    assert np.array_equal(hb[: oc.h_len], oc.hbits()) and not hb[oc.h_len:].any()
    a, b, c = oc.products()
    rows = s["constraints"]
    assert np.array_equal(prod[:rows], a) and np.array_equal(prod[rows:2 * rows], b)
    assert np.array_equal(prod[2 * rows:], c)


def test_false_statement_is_unsatisfied():
    inp, out, _ = ci.instance("sha256-chain", 1, 4)
    bad = out.copy()
    bad[17] ^= 1
    ps = bz.CircuitProofSystem("sha256-chain", inp, bad, 100)
    with pytest.raises(bz.BitzError) as e:
        ps.prove()
    assert e.value.code == "Unsatisfied"
    rc, _, _ = of.prove(1, inp, bad, 100)
    assert rc == 3


def test_per_round_launches_give_the_same_proof():
    """BITZ_RESIDENT_ROUNDS=0 runs the GKR tail rounds as separate launches
    instead of one resident kernel; the proof bytes must not change."""
    import os
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import bitz_b200 as bz\n"
            "from bitz_b200 import statements as ci\n"
            "inp, out, _ = ci.instance('sha256-chain', 2, 13)\n"
            "p, _ = bz.CircuitProofSystem('sha256-chain', inp, out, 100).prove()\n"
            "sys.stdout.write(p.hex())\n") % os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    runs = []
    for flag in ("0", "1"):
        env = dict(os.environ, BITZ_RESIDENT_ROUNDS=flag)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        runs.append(r.stdout)
    assert runs[0] == runs[1] and len(runs[0]) > 1000


@pytest.mark.parametrize("kind,blocks,seed,security", [
    ("sha256-chain", 64, 1, 100),        # the benchmark statement
    ("sha256-block-aligned", 32, 3, 100),
    ("sha256-2kb", 32, 4, 128),
])
def test_full_size_proofs_are_accepted_by_the_restated_verifier(kind, blocks, seed, security):
    inp, out, _ = ci.instance(kind, blocks, seed)
    proof, _ = bz.CircuitProofSystem(kind, inp, out, security).prove()
    assert of.verify(ci.KINDS[kind], inp, out, security, proof) == 0
    bad = bytearray(proof)
    bad[len(bad) // 2] ^= 0x10
    assert of.verify(ci.KINDS[kind], inp, out, security, bytes(bad)) != 0


def test_large_proof_is_accepted_by_the_restated_verifier():
    """sha256-chain n=1024 at 128 bits (unique decoding, no OOD): a
    multi-million-entry witness, checked by the verifier instead of a second
    proof on the CPU."""
    inp, out, _ = ci.instance("sha256-chain", 1024, 2)
    proof, _ = bz.CircuitProofSystem("sha256-chain", inp, out, 128).prove()
    assert of.verify(ci.KINDS["sha256-chain"], inp, out, 128, proof) == 0
