"""Benchmark: SHA-256 blocks proven per second on B200.

Workload: sha256-chain, 64 blocks of uniform random bytes from SplitMix64 seed 1,
standard IV, PCS security 100 (list decoding + OOD). One step is one complete
proof: witness, commitment and prove (tooling/cli/src/benchmark.rs:28-79
times the same three stages). Setup (constraint synthesis, matrix digest) is
done once per statement and excluded, as in the reference's benchmark. The L2
cache is flushed before every timed proof.

Beside it, the batched workload: 256 independent sha256-block-aligned proofs
with message lengths uniform over 0..32 blocks (SplitMix64 seed 3), proved on
concurrent prover lanes, against the same 256 proved one after another.

``--serve`` instead runs the serving workload: an open-loop Poisson stream of
requests (half sha256-2kb, half block-aligned with log-uniform 1..512 blocks,
seed 4) into the prove server, sweeping the arrival rate, and prints one JSON
line per rate with p50/p99 latency and blocks/s.

Multi-GPU: one process per GPU (torchrun), each proving its own statements,
no collective on the data path ("replicas"): value = all proofs' blocks / the
slowest rank's time.

``--impl reference`` times the CPU restatement of the reference prover
(oracle/, the reference is Rust and cannot be built here) on the host cores.
"""
import argparse
import json
import os
import random
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
PROBED_KERNEL = "gkr_bind_sums"
# per-launch DRAM traffic of the probed kernel, from the ncu capture summarised here
TRAFFIC_SUMMARY = os.path.join(ROOT, "profiles", "gkr_bind_sums_sha256-chain-n64.md")


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
    p.add_argument("--lanes", type=int, default=16)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--serve", action="store_true")
    p.add_argument("--serve-requests", type=int, default=96)
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
    from bitz_b200 import statements
    return statements.blocks_proven(args.circuit, n_inputs)


def peaks():
    try:
        return json.load(open(MEASURED_PEAKS)), "measured"
    except Exception:
        return {"hbm_gbs": FALLBACK_HBM_GBS}, "fallback"


def profile_figure(key):
    """A figure of the probed kernel's ncu summary (e.g. DRAM bytes per
    launch), or None."""
    try:
        for line in open(TRAFFIC_SUMMARY):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(q * len(xs)))]


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
        list(ex.map(one, range(args.steps)))
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


def batched(args, bz):
    """256 sha256-block-aligned proofs, k ~ U{0..32} (seed 3): sequential on
    one lane against concurrent on ``args.lanes`` lanes."""
    from bitz_b200 import statements
    mix = statements.batch_mix(3, 256, 32)
    systems = [bz.CircuitProofSystem(kind, inp, out, args.security) for kind, inp, out in mix]
    blocks = sum(statements.blocks_proven(kind, inp.size) for kind, inp, _ in mix)
    # warm-up: every lane's scratch grows to the largest shape of the mix
    largest = sorted(range(len(mix)), key=lambda i: -mix[i][1].size)[:args.lanes]
    bz.batch_prove([systems[i] for i in largest], args.lanes)
    bz.batch_prove([systems[largest[0]]], 1)
    bz.batch_prove(systems, args.lanes)
    res = {}
    for name, lanes in (("sequential", 1), ("batched", args.lanes)):
        bz.l2_flush()
        t0 = time.perf_counter()
        proofs, lat = bz.batch_prove(systems, lanes)
        wall = time.perf_counter() - t0
        res[name] = (blocks / wall, lat, proofs)
    same = res["sequential"][2] == res["batched"][2]
    return {"workload": "256 x sha256-block-aligned, k ~ U{0..32} blocks (SplitMix64 seed 3), "
                        f"pcs-security-bits {args.security}",
            "blocks": blocks, "lanes": args.lanes,
            "value": res["batched"][0], "unit": "blocks/s",
            "sequential_value": res["sequential"][0],
            "speedup_vs_sequential": res["batched"][0] / res["sequential"][0],
            "latency_ms": {"p50": pct(res["batched"][1], 0.5), "p99": pct(res["batched"][1], 0.99)},
            "sequential_latency_ms": {"p50": pct(res["sequential"][1], 0.5),
                                      "p99": pct(res["sequential"][1], 0.99)},
            "proofs_identical_to_sequential": same}


def serve(args):
    """Open-loop Poisson arrivals into the prove server, rate swept upward
    until p99 latency exceeds 10x the single-proof latency."""
    import bitz_b200 as bz
    from bitz_b200 import statements
    bz.set_device(dist_env()[2])
    mix = statements.serve_mix(4, args.serve_requests, 512)
    blocks = [statements.blocks_proven(k, i.size) for k, i, _ in mix]
    # circuit shapes are built once per (circuit, size) and cached, as the
    # reference's benchmark excludes setup: build every shape of the stream
    t0 = time.perf_counter()
    shapes = {}
    for kind, inp, out in mix:
        shapes.setdefault((kind, inp.size), (kind, inp, out))
    prove_only, alone = [], []
    for kind, inp, out in shapes.values():
        ps = bz.CircuitProofSystem(kind, inp, out, args.security)
        ps.prove()
    setup_s = time.perf_counter() - t0
    # proof bytes and prove-only latency of the first requests, alone
    for kind, inp, out in mix[:16]:
        ps = bz.CircuitProofSystem(kind, inp, out, args.security)
        t = time.perf_counter()
        p, _ = ps.prove()
        prove_only.append(1000 * (time.perf_counter() - t))
        alone.append(p)
    rng = random.Random(4)
    with bz.ProveServer(lanes=args.lanes, hbm_budget=96 << 30, security_bits=args.security) as srv:
        # warm-up: every lane's scratch grows to the largest shape of the stream
        big = max(mix, key=lambda m: m[1].size)
        warm = [srv.submit(*big) for _ in range(args.lanes)]
        for t in warm:
            while srv.poll(t, 50) is None:
                pass
        # single-request latency: each of the first requests alone on an idle
        # server, submit to proof bytes (statement preparation included)
        alone_served = []
        for kind, inp, out in mix:
            t = srv.submit(kind, inp, out)
            r = None
            while r is None:
                r = srv.poll(t, 50)
            alone_served.append(r[1])
        # the mix is uneven (1..512 blocks), so the single-request bar for the
        # sweep is the p99 of the requests served one at a time
        single = pct(alone_served, 0.99)
        rate = 1000.0 / statistics.mean(alone_served)  # one request at a time
        while True:
            gaps = [rng.expovariate(rate) for _ in mix]
            tickets, t0 = [], time.perf_counter()
            due = t0
            for (kind, inp, out), g in zip(mix, gaps):
                due += g
                while time.perf_counter() < due:
                    time.sleep(min(0.0005, max(0.0, due - time.perf_counter())))
                tickets.append(srv.submit(kind, inp, out))
            lat, got = [], {}
            while len(got) < len(tickets):
                for t in tickets:
                    if t not in got:
                        r = srv.poll(t, 2)
                        if r is not None:
                            got[t] = r
            wall = time.perf_counter() - t0
            lat = [got[t][1] for t in tickets]
            same = all(got[t][0] == a for t, a in zip(tickets[:16], alone))
            p99 = pct(lat, 0.99)
            print(json.dumps({"metric": "SHA-256 blocks proven/sec (serving)", "rate_rps": rate,
                              "value": sum(blocks) / wall, "unit": "blocks/s",
                              "latency_ms": {"p50": pct(lat, 0.5), "p99": p99},
                              "single_request_latency_ms": {
                                  "p50": pct(alone_served, 0.5), "p99": single},
                              "prove_only_latency_ms": statistics.median(prove_only),
                              "lanes": args.lanes,
                              "requests": len(mix), "peak_in_flight": srv.stats()["peak_in_flight"],
                              "shapes_prebuilt": len(shapes), "setup_s": setup_s,
                              "proofs_identical_to_alone": same,
                              "workload": "Poisson arrivals; 50% sha256-2kb, 50% sha256-block-aligned "
                                          "k = floor(2^U(0,9)) in 1..512 (seed 4)"}), flush=True)
            if p99 > 10 * single or rate > 2000:
                break
            rate *= 1.5


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
    # device-resident timed region: the statement stays staged, the L2 is
    # flushed before every proof, each proof timed by CUDA events on its stream
    dist.barrier()
    launches0 = bz.launch_count()
    with Clocks(local) as clk:
        spans = []
        for _ in range(args.steps):
            bz.l2_flush()
            proof, times = ps.prove(restage=False)
            spans.append(times["device_ms"])
    launches = bz.launch_count() - launches0
    dist.barrier()
    # the probed kernel timed alone, in a pass of its own: with the probe on,
    # its rounds run as separate launches instead of queued behind one another
    # (a queued round kernel's last block also waits for the next challenge)
    bz.probe_kernel(PROBED_KERNEL)
    probe_spans = []
    for _ in range(min(args.steps, 3)):
        bz.l2_flush()
        _, ptimes = ps.prove(restage=False)
        probe_spans.append(ptimes["device_ms"])
    probe_ms, probe_bytes, probe_launches = bz.probe_read()
    bz.probe_kernel(None)
    dist.barrier()
    dev_total_ms = dist.max(sum(spans))
    # end to end through the C ABI: the statement copied from host memory and
    # the proof bytes returned to host memory on every step
    dist.barrier()
    e2e_s = 0.0
    for _ in range(args.steps):
        bz.l2_flush()
        t1 = time.perf_counter()
        proof, _ = ps.prove(restage=True)
        e2e_s += time.perf_counter() - t1
    e2e_s = dist.max(e2e_s)
    dist.barrier()
    value = world * blocks * args.steps / (dev_total_ms / 1000.0)
    e2e = world * blocks * args.steps / e2e_s
    stats = ps.stats()
    h2d = 4 * (8 + 16) * stats["compressions"] + 8 * stats["compressions"] + (inputs.size + 7) // 8 \
        + inputs.size + 256
    batch = None
    if world == 1 and not args.no_batch:
        batch = batched(args, bz)
    line = None
    if rank == 0:
        pk, pk_kind = peaks()
        achieved = probe_bytes / (probe_ms / 1000.0) / 1e9 if probe_ms > 0 else None
        per_launch = profile_figure("traffic_bytes_per_launch")
        line = {
            "metric": "SHA-256 blocks proven/sec", "value": value, "unit": "blocks/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(spans),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "gf2^128+fp121", "data": f"synthetic (SplitMix64 seed {args.seed})",
            "config": {"workload": f"{args.circuit} n={args.blocks} pcs-security-bits {args.security}",
                       "parallelism": f"replicas x{world}", "seed": args.seed,
                       "step": "one proof: witness + commit + prove",
                       "l2": "flushed (256 MiB device write) before every timed proof"},
            "latency_ms": {"p50": statistics.median(spans), "p99": pct(spans, 0.99)},
            "stage_ms": {k: times[k] for k in ("witness_ms", "commit_ms", "prove_ms")},
            "e2e": {"value": e2e, "unit": "blocks/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": len(proof)},
            "gpu_launches": launches,
            "roofline": {"kernel": PROBED_KERNEL, "bound": "hbm", "achieved": achieved,
                         "peak": pk["hbm_gbs"], "peak_source": f"hbm_gbs, {pk_kind}", "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"] if achieved else None,
                         "traffic": per_launch,
                         "algorithmic_bytes_per_launch": probe_bytes / probe_launches if probe_launches else None,
                         "launches": probe_launches,
                         "avg_launch_us": 1000 * probe_ms / probe_launches if probe_launches else None,
                         "share_of_device_time": probe_ms / sum(probe_spans) if probe_spans else None,
                         "integer_issue_active_ncu": profile_figure("issue_active_largest_launch"),
                         "note": "integer-issue bound (GF(2^128) products), not HBM bound: "
                                 "see profiles/gkr_bind_sums_sha256-chain-n64.md"},
            "clocks": clk.summary(),
            "proof_bytes": len(proof),
            "peaks": pk_kind,
        }
        if batch:
            line["batched"] = batch
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args, inputs, outputs, blocks)
        print(json.dumps(line))
    dist.close()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.serve:
        serve(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
