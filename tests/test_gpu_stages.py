"""The reference's staged API: CircuitProofSystem::witness, commit and prove
(tooling/cli/src/end_to_end.rs:215-336) as separate C-ABI calls give the same
proof bytes as the single call, and misuse fails with the reference's errors."""
import pytest

import bitz_b200 as bz
from bitz_b200 import statements as ci

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,blocks,seed,security", [
    ("sha256-chain", 3, 21, 100), ("sha256-block-aligned", 2, 22, 128),
    ("sha256-chain", 64, 1, 100)])
def test_staged_calls_give_the_single_call_proof(kind, blocks, seed, security):
    inp, out, _ = ci.instance(kind, blocks, seed)
    ps = bz.CircuitProofSystem(kind, inp, out, security)
    single, _ = ps.prove()
    wit = ps.witness(inp)
    com = ps.commit(wit)
    staged, _ = ps.prove(wit, com)
    assert staged == single
    # the system proves again afterwards, both ways
    assert ps.prove()[0] == single
    w2 = ps.witness(inp)
    assert ps.prove(w2, ps.commit(w2))[0] == single


def test_staged_proofs_of_two_systems_interleave():
    """Two staged proofs held at once: one on the default lane, one on a pool
    lane; a single-call proof of a third system in between takes a free lane."""
    stmts = [ci.instance("sha256-chain", 2, 30 + i) for i in range(3)]
    systems = [bz.CircuitProofSystem("sha256-chain", i, o, 100) for i, o, _ in stmts]
    alone = [s.prove()[0] for s in systems]
    w0 = systems[0].witness(stmts[0][0])
    w1 = systems[1].witness(stmts[1][0])
    c1 = systems[1].commit(w1)
    c0 = systems[0].commit(w0)
    assert systems[2].prove()[0] == alone[2]
    assert systems[1].prove(w1, c1)[0] == alone[1]
    assert systems[0].prove(w0, c0)[0] == alone[0]


def test_staged_misuse_is_reported():
    inp, out, _ = ci.instance("sha256-chain", 1, 40)
    ps = bz.CircuitProofSystem("sha256-chain", inp, out, 100)
    with pytest.raises(bz.BitzError) as e:  # end_to_end.rs:216-218
        ps.witness(inp[:-512] if inp.size > 512 else inp[:100])
    assert "wrong witness input length" in str(e.value)
    bad = inp.copy()
    bad[5] ^= 1
    with pytest.raises(bz.BitzError) as e:  # inputs that do not satisfy the statement
        ps.witness(bad)
    assert e.value.code == "Unsatisfied"
    w = ps.witness(inp)
    with pytest.raises(bz.BitzError):  # one staged proof per system
        ps.witness(inp)
    with pytest.raises(bz.BitzError):  # the single call refuses while one is staged
        ps.prove()
    c = ps.commit(w)
    with pytest.raises(bz.BitzError):  # committed twice
        ps.commit(w)
    del c, w  # dropping the handles ends the staged proof
    import gc
    gc.collect()
    assert ps.prove()[0] == ps.prove()[0]
