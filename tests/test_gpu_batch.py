"""Batched and served proving: every proof made in a mix of concurrent
proofs on several lanes is byte-identical to the same statement proved alone,
and to the oracle's proof for the small statements."""
import time

import numpy as np
import pytest

import bitz_b200 as bz
from bitz_b200 import statements as ci
from oracle import ffi as of

pytestmark = pytest.mark.gpu

# uneven sizes and kinds, empty message included
MIX = [("sha256-block-aligned", 0), ("sha256-chain", 3), ("sha256-block-aligned", 2),
       ("sha256-compression", 1), ("sha256-block-aligned", 5), ("sha256-chain", 1),
       ("sha256-2kb", 32), ("sha256-block-aligned", 1)]


def statement(i, kind, blocks):
    st = ci.random_state(40 + i) if kind == "sha256-compression" else None
    return ci.instance(kind, blocks, 300 + i, st)[:2]


@pytest.fixture(scope="module")
def alone():
    """Each statement proved alone on the default lane."""
    out = []
    for i, (kind, blocks) in enumerate(MIX):
        inp, outp = statement(i, kind, blocks)
        proof, _ = bz.CircuitProofSystem(kind, inp, outp, 100).prove()
        out.append(proof)
    return out


def test_alone_matches_oracle_for_small_statements(alone):
    of.lib().o_set_clmul_mode(1)
    try:
        for i, (kind, blocks) in enumerate(MIX):
            if kind == "sha256-2kb" or blocks > 3:
                continue
            inp, outp = statement(i, kind, blocks)
            rc, oproof, _ = of.prove(ci.KINDS[kind], inp, outp, 100)
            assert rc == 0
            assert oproof == alone[i], (kind, blocks)
    finally:
        of.lib().o_set_clmul_mode(0)


@pytest.mark.parametrize("lanes", [1, 3, 8])
def test_batch_matches_alone(alone, lanes):
    systems = [bz.CircuitProofSystem(kind, *statement(i, kind, blocks), 100)
               for i, (kind, blocks) in enumerate(MIX)]
    proofs, lat = bz.batch_prove(systems, lanes)
    assert proofs == alone
    assert all(x > 0 for x in lat)


def _batch_in_child(env_updates):
    """The MIX proved twice on eight lanes in a child process with the given
    environment (the library reads these settings once per process)."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    code = ("import sys; sys.path[:0] = [%r, %r]\n"
            "from test_gpu_batch import MIX, statement\n"
            "import bitz_b200 as bz\n"
            "systems = [bz.CircuitProofSystem(k, *statement(i, k, b), 100) "
            "for i, (k, b) in enumerate(MIX)]\n"
            "proofs, lat = bz.batch_prove(systems, 8)\n"
            "again, _ = bz.batch_prove(systems, 8)\n"
            "assert again == proofs\n"
            "sys.stdout.write(''.join(p.hex() + '\\n' for p in proofs))\n") % (
                here, os.path.dirname(here))
    env = dict(os.environ, **env_updates)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=600, cwd=here)
    assert r.returncode == 0, r.stderr[-3000:]
    return [bytes.fromhex(x) for x in r.stdout.split()]


def test_lanes_sharing_host_threads_as_fibers(alone):
    """Eight lanes on two host threads (four fibers each, switching wherever a
    lane waits for the device): the same proofs."""
    assert _batch_in_child({"BITZ_LANE_THREADS": "2"}) == alone


def test_pooled_lanes_with_resident_middle_rounds(alone):
    """Pooled lanes with their GKR, Spartan and post-GKR middle rounds in
    32-block resident grids (BITZ_POOL_MID=1) instead of queued launches: the
    same proofs."""
    assert _batch_in_child({"BITZ_POOL_MID": "1"}) == alone


def test_batch_twice_on_the_same_systems(alone):
    systems = [bz.CircuitProofSystem(kind, *statement(i, kind, blocks), 100)
               for i, (kind, blocks) in enumerate(MIX)]
    first, _ = bz.batch_prove(systems, 4)
    second, _ = bz.batch_prove(systems, 4)
    assert first == second == alone


def test_batch_reports_a_false_statement():
    inp, outp = statement(0, "sha256-chain", 2)
    bad = outp.copy()
    bad[5] ^= 1
    good = bz.CircuitProofSystem("sha256-chain", inp, outp, 100)
    wrong = bz.CircuitProofSystem("sha256-chain", inp, bad, 100)
    with pytest.raises(bz.BitzError) as e:
        bz.batch_prove([good, wrong], 2)
    assert e.value.code == "Unsatisfied"


def drain(srv, tickets, timeout_s=120):
    res = {}
    t0 = time.time()
    while len(res) < len(tickets) and time.time() - t0 < timeout_s:
        for t in tickets:
            if t not in res:
                r = srv.poll(t, wait_ms=5)
                if r is not None:
                    res[t] = r
    assert len(res) == len(tickets)
    return [res[t] for t in tickets]


def test_server_mix_matches_alone(alone):
    with bz.ProveServer(lanes=4, hbm_budget=64 << 30) as srv:
        tickets = []
        for i, (kind, blocks) in enumerate(MIX):
            tickets.append(srv.submit(kind, *statement(i, kind, blocks)))
        got = drain(srv, tickets)
        st = srv.stats()
    assert [p for p, _ in got] == alone
    assert st["submitted"] == st["finished"] == len(MIX)
    assert st["in_flight"] == 0 and st["queued"] == 0
    assert st["peak_in_flight"] >= 2


def test_server_budget_admits_one_at_a_time(alone):
    # a budget below every footprint: one request in flight at a time
    with bz.ProveServer(lanes=4, hbm_budget=1) as srv:
        tickets = [srv.submit(kind, *statement(i, kind, blocks))
                   for i, (kind, blocks) in enumerate(MIX[:4])]
        got = drain(srv, tickets)
        st = srv.stats()
    assert [p for p, _ in got] == alone[:4]
    assert st["peak_in_flight"] == 1


def test_server_requests_arriving_while_others_run(alone):
    with bz.ProveServer(lanes=3) as srv:
        first = [srv.submit(kind, *statement(i, kind, blocks))
                 for i, (kind, blocks) in enumerate(MIX[:3])]
        time.sleep(0.002)
        later = [srv.submit(kind, *statement(i, kind, blocks))
                 for i, (kind, blocks) in enumerate(MIX) if i >= 3]
        got = drain(srv, first + later)
    assert [p for p, _ in got] == alone
    assert all(lat > 0 for _, lat in got)


def test_server_failure_is_reported_per_request(alone):
    inp, outp = statement(1, "sha256-chain", 3)
    bad = outp.copy()
    bad[0] ^= 1
    with bz.ProveServer(lanes=2) as srv:
        tb = srv.submit("sha256-chain", inp, bad)
        tg = srv.submit("sha256-chain", inp, outp)
        with pytest.raises(bz.BitzError):
            while srv.poll(tb, wait_ms=50) is None:
                pass
        r = None
        while r is None:
            r = srv.poll(tg, wait_ms=50)
    assert r[0] == alone[1]
