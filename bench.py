"""Benchmark: SHA-256 blocks proven per second on B200.

Workload: sha256-chain, 64 blocks of uniform random bytes from SplitMix64 seed 1,
standard IV, PCS security 100 (list decoding + OOD). One step is one complete
proof: witness, commitment and prove (tooling/cli/src/benchmark.rs:28-79
times the same three stages). Setup (constraint synthesis, matrix digest) is
done once per statement and excluded, as in the reference's benchmark.

Multi-GPU: one process per GPU (torchrun), each proving its own statements,
no collective on the data path ("replicas"): value = all proofs' blocks / the
slowest rank's time.

``--impl reference`` times the CPU restatement of the reference prover
(oracle/, the reference is Rust and cannot be built here) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--circuit", default="sha256-chain")
    p.add_argument("--blocks", type=int, default=64)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--security", type=int, default=100)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Dist:
    """Barrier and max-reduce across ranks (gloo over host tensors)."""

    def __init__(self, world):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.stop = threading.Event()
        self.th = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def statement(args):
    from bitz_b200 import statements
    return statements.instance(args.circuit, args.blocks, args.seed)


def blocks_proven(args, n_inputs):
    """Compression blocks per proof: message blocks, plus the padding block for
    the block-aligned circuits."""
    if args.circuit in ("sha256-block-aligned", "sha256-2kb"):
        return n_inputs // 512 + 1
    return max(n_inputs // 512, 1)


def peaks():
    try:
        return json.load(open(MEASURED_PEAKS)), "measured"
    except Exception:
        return {"hbm_gbs": FALLBACK_HBM_GBS}, "fallback"


def cpu_baseline(args, inputs, outputs, blocks):
    """One complete proof of the same statement with the CPU restatement of the
    reference prover, single-threaded, with the reference's x86 GF(2^128)
    kernel (a per-bit carryless multiply, crates/field/src/gf128/portable.rs)."""
    from oracle import ffi as of
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    of.lib().o_set_clmul_mode(0)
    kinds = {"sha256-compression": 0, "sha256-chain": 1, "sha256-block-aligned": 2, "sha256-2kb": 3}
    rc, proof, times = of.prove(kinds[args.circuit], inputs, outputs, args.security)
    if rc != 0:
        raise RuntimeError(f"oracle prover failed: {rc}")
    secs = float(times[1] + times[2])  # commit + prove, total_prove_ms of benchmark.rs:97
    return {"value": blocks / secs, "unit": "blocks/s", "cores": 1, "kind": "port",
            "sample": f"one {args.circuit} n={blocks} proof (commit + prove {secs:.1f} s; "
                      f"witness replay {times[0]:.1f} s reported apart), portable bit-loop GF(2^128) "
                      "multiply as the reference's x86 kernel, 1 thread"}


def reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor

    from oracle import ffi as of
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    of.lib().o_set_clmul_mode(0)
    inputs, outputs, _ = statement(args)
    blocks = blocks_proven(args, inputs.size)
    kinds = {"sha256-compression": 0, "sha256-chain": 1, "sha256-block-aligned": 2, "sha256-2kb": 3}
    cores = os.cpu_count() or 1

    def one(_):
        t = time.perf_counter()
        rc, _, times = of.prove(kinds[args.circuit], inputs, outputs, args.security)
        assert rc == 0
        return time.perf_counter() - t, float(times[1] + times[2])

    with ThreadPoolExecutor(max_workers=cores) as ex:
        list(ex.map(one, range(args.warmup)))
        t0 = time.perf_counter()
        res = list(ex.map(one, range(args.steps)))
        wall = time.perf_counter() - t0
    value = blocks * args.steps / wall
    line = {"impl": "reference", "metric": "SHA-256 blocks proven/sec", "value": value,
            "unit": "blocks/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "gf2^128+fp121", "data": f"synthetic (SplitMix64 seed {args.seed})",
            "config": {"workload": f"{args.circuit} n={args.blocks} pcs-security-bits {args.security}",
                       "seed": args.seed},
            "cpu_baseline": {"value": value, "unit": "blocks/s", "cores": min(cores, args.steps),
                             "kind": "port",
                             "sample": f"{args.steps} proofs on {min(cores, args.steps)} threads of the "
                                       "CPU restatement (oracle/), witness replay + commit + prove each"},
            "e2e": {"value": value, "unit": "blocks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def ours(args):
    world, rank, local = dist_env()
    import bitz_b200 as bz
    lib_path = os.path.join(ROOT, "bitz_b200", "libbitz_b200.so")
    if not os.path.exists(lib_path):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "bitz_b200")], check=True)
    dist = Dist(world)
    bz.set_device(local)
    inputs, outputs, _ = statement(args)
    blocks = blocks_proven(args, inputs.size)
    ps = bz.CircuitProofSystem(args.circuit, inputs, outputs, args.security)
    for _ in range(args.warmup):
        ps.prove(restage=False)
    # device-resident timed region
    dist.barrier()
    launches0 = bz.launch_count()
    with Clocks(local) as clk:
        spans = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            proof, times = ps.prove(restage=False)
            spans.append(times["device_ms"])
        wall = time.perf_counter() - t0
    launches = bz.launch_count() - launches0
    dist.barrier()
    dev_total_ms = dist.max(sum(spans))
    # end to end through the C ABI: the statement copied from host memory and
    # the proof bytes returned to host memory on every step
    dist.barrier()
    t1 = time.perf_counter()
    for _ in range(args.steps):
        proof, _ = ps.prove(restage=True)
    e2e_wall = dist.max(time.perf_counter() - t1)
    dist.barrier()
    value = world * blocks * args.steps / (dev_total_ms / 1000.0)
    e2e = world * blocks * args.steps / e2e_wall
    stats = ps.stats()
    h2d = 4 * (8 + 16) * stats["compressions"] + 8 * stats["compressions"] + (inputs.size + 7) // 8 \
        + inputs.size + 256
    line = None
    if rank == 0:
        pk, pk_kind = peaks()
        line = {
            "metric": "SHA-256 blocks proven/sec", "value": value, "unit": "blocks/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(spans),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "gf2^128+fp121", "data": f"synthetic (SplitMix64 seed {args.seed})",
            "config": {"workload": f"{args.circuit} n={args.blocks} pcs-security-bits {args.security}",
                       "parallelism": f"replicas x{world}", "seed": args.seed,
                       "step": "one proof: witness + commit + prove",
                       "l2": "every proof re-reads its tables; working set per proof below L2 at n=64"},
            "latency_ms": {"p50": statistics.median(spans),
                           "p99": sorted(spans)[min(len(spans) - 1, int(0.99 * len(spans)))]},
            "stage_ms": {k: times[k] for k in ("witness_ms", "commit_ms", "prove_ms")},
            "e2e": {"value": e2e, "unit": "blocks/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": len(proof)},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "proof_bytes": len(proof),
            "peaks": pk_kind,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args, inputs, outputs, blocks)
        print(json.dumps(line))
    dist.close()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
