"""The multi-GPU path of bench.py: one process per GPU, each proving its own
statements with no collective on the data path; the ranks only meet at
barriers and in the max of their timings (gloo over host tensors). Two gloo
ranks on CPU exercise that plumbing; no GPU is needed."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_env() == (world, rank, rank)
    d = bench.Dist(world)
    d.barrier()
    # each rank's device time differs; the job's time is the slowest rank's
    slowest = d.max(10.0 + rank * 5.0)
    d.barrier()
    d.close()
    results[rank] = slowest


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        results = m.dict()
        mp.start_processes(_rank, args=(world, port, results), nprocs=world, start_method="spawn")
        assert dict(results) == {0: 15.0, 1: 15.0}


def test_replica_value_counts_every_rank():
    """value = all ranks' blocks / the slowest rank's time (weak scaling)."""
    import bench
    assert bench.replica_value(world=2, blocks=64, steps=10, slowest_ms=100.0) == 2 * 64 * 10 / 0.1
