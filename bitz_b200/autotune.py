"""Chooses the batched prover's lane count and host-thread cap on this machine.

Batched proving runs L prover lanes (one CUDA stream each) driven by at most T
host threads, lanes beyond T sharing threads as fibers. The best (L, T)
depends on the GPU, the host's cores and the workload's statement sizes. This
script proves a workload (by default the 256-statement block-aligned mix,
k ~ U{0..32}, SplitMix64 seed 3) at every (L, T) of a grid, each in a fresh
process (T is read once per process), checks the proofs of every run against
the first run's, and writes the fastest to bitz_b200/tuning.json:

    {"lanes": L, "lane_threads": T, "blocks_per_s": ..., "gpu": ..., "grid": [...]}

``bitz_b200.batch_prove`` uses the table's lane count when called without
one, and the package sets BITZ_LANE_THREADS from it unless the environment
sets it. Run on the machine that will prove:

    python -m bitz_b200.autotune [--lanes 8,16,24,32,48] [--threads 4,8,0] [--repeats 2]

(threads 0 stands for the host's hardware thread count).
"""
import argparse
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")

_CHILD = r"""
import hashlib, json, sys, time
sys.path.insert(0, %(root)r)
import bitz_b200 as bz
from bitz_b200 import statements
mix = statements.batch_mix(%(seed)d, %(count)d, %(max_blocks)d)
systems = [bz.CircuitProofSystem(k, i, o, %(security)d) for k, i, o in mix]
blocks = sum(statements.blocks_proven(k, i.size) for k, i, _ in mix)
bz.batch_prove(systems, %(lanes)d)  # warm-up: every lane's scratch grown
best, digest = 0.0, None
for _ in range(%(repeats)d):
    t0 = time.perf_counter()
    proofs, _ = bz.batch_prove(systems, %(lanes)d)
    best = max(best, blocks / (time.perf_counter() - t0))
    d = hashlib.sha256(b"".join(proofs)).hexdigest()
    assert digest in (None, d), "proofs changed between runs"
    digest = d
print(json.dumps({"blocks_per_s": best, "proofs_sha256": digest}))
"""


def run_point(lanes, threads, args):
    env = dict(os.environ)
    env.pop("BITZ_LANE_THREADS", None)
    if threads:
        env["BITZ_LANE_THREADS"] = str(threads)
    code = _CHILD % {"root": os.path.dirname(HERE), "seed": args.seed, "count": args.count,
                     "max_blocks": args.max_blocks, "security": args.security, "lanes": lanes,
                     "repeats": args.repeats}
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=args.timeout)
    if r.returncode != 0:
        raise RuntimeError(f"lanes={lanes} threads={threads}: {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


def main():
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--lanes", default="8,16,24,32,48")
    p.add_argument("--threads", default="4,8,0")
    p.add_argument("--repeats", type=int, default=2)
    p.add_argument("--seed", type=int, default=3)
    p.add_argument("--count", type=int, default=256)
    p.add_argument("--max-blocks", type=int, default=32)
    p.add_argument("--security", type=int, default=100)
    p.add_argument("--timeout", type=int, default=600)
    p.add_argument("--out", default=TABLE)
    args = p.parse_args()
    hw = os.cpu_count() or 1
    grid, digest, best = [], None, None
    for t in (int(x) for x in args.threads.split(",")):
        threads = t or hw
        for lanes in (int(x) for x in args.lanes.split(",")):
            res = run_point(lanes, threads, args)
            if digest is None:
                digest = res["proofs_sha256"]
            if res["proofs_sha256"] != digest:
                raise RuntimeError(f"lanes={lanes} threads={threads}: different proofs")
            point = {"lanes": lanes, "lane_threads": threads, "blocks_per_s": res["blocks_per_s"]}
            grid.append(point)
            print(json.dumps(point), flush=True)
            if best is None or point["blocks_per_s"] > best["blocks_per_s"]:
                best = point
    try:
        gpu = subprocess.run(["nvidia-smi", "--query-gpu=name", "--format=csv,noheader", "-i", "0"],
                             capture_output=True, text=True, timeout=30).stdout.strip() or None
    except Exception:
        gpu = None
    table = dict(best, host_threads=hw, gpu=gpu,
                 workload=f"batch_mix(seed={args.seed}, count={args.count}, "
                          f"max_blocks={args.max_blocks}), pcs-security-bits {args.security}",
                 proofs_sha256=digest, grid=grid)
    with open(args.out, "w") as f:
        json.dump(table, f, indent=1)
    print(json.dumps({k: v for k, v in table.items() if k != "grid"}))


if __name__ == "__main__":
    main()
