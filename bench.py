"""Benchmark: SHA-256 blocks proven per second on B200.

Workload: sha256-chain, 64 blocks of uniform random bytes from SplitMix64 seed 1,
standard IV, PCS security 100 (list decoding + OOD). One step is one complete
proof: witness, commitment and prove (tooling/cli/src/benchmark.rs:28-79
times the same three stages). Setup (constraint synthesis, matrix digest) is
done once per statement and excluded, as in the reference's benchmark. The L2
cache is flushed before every timed proof.

Beside it, in the same JSON line:
- ``batched``: 256 independent sha256-block-aligned proofs with message lengths
  uniform over 0..32 blocks (SplitMix64 seed 3), proved on concurrent prover
  lanes, against the same 256 proved one after another by the plain
  single-proof call;
- ``large``: sha256-chain n=1024 at PCS security 128 (seed 2);
- ``serving``: an open-loop Poisson stream of requests (half sha256-2kb, half
  block-aligned with log-uniform 1..512 blocks, seed 4) into the prove server,
  the arrival rate swept upward, against the same stream proved one request
  after another;
- ``roofline``: the kernel with the largest share of a proof's device time,
  every launch timed with CUDA events, held to the measured HBM bandwidth and
  the measured GF(2^128) product throughput of the GPU.

``--serve`` runs the serving sweep alone, one JSON line per rate.

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
PROFILES = os.path.join(ROOT, "profiles")


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
    p.add_argument("--lanes", type=int, default=None,
                   help="prover lanes for the batched and serving workloads (default: the "
                        "tuned count of bitz_b200/tuning.json, else 16)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--serve", action="store_true")
    p.add_argument("--serve-requests", type=int, default=96)
    p.add_argument("--serving-requests", type=int, default=96,
                   help="requests in the default line's serving sweep")
    p.add_argument("--serving-rates", type=int, default=10,
                   help="arrival rates at most in the default line's serving sweep")
    p.add_argument("--no-large", action="store_true")
    p.add_argument("--no-serving", action="store_true")
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


def profile_figure(summary, key, tag="sha256-chain-n64"):
    """A figure (e.g. DRAM bytes per launch) from a committed ncu summary of
    a workload, or None: the lines ``key: value`` of profiles/<summary>_<tag>.md."""
    path = os.path.join(PROFILES, f"{summary}_{tag}.md")
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def roofline(bz, ps, steps, hbm_gbs, pk_kind, tag="sha256-chain-n64"):
    """Times every launch of the instrumented kernels with CUDA events over
    ``steps`` proofs (every round its own launch, as under a kernel profiler),
    picks the kernel with the largest share of the proofs' device time, and
    holds it to its roofline: its algorithmic bytes at the measured HBM
    bandwidth and its GF(2^128) products at the GPU's measured product
    throughput (bitz_diag_gf_peak), whichever takes longer."""
    peaks = {k: bz.gf_peak(i) for i, k in enumerate(("gmuls", "wides", "tables"))}
    bz.probe_kernel("*")
    spans = []
    for _ in range(steps):
        bz.l2_flush()
        _, t = ps.prove(restage=False)
        spans.append(t["device_ms"])
    table = {k: bz.probe_read(k) for k in bz.probe_kernels()}
    bz.probe_kernel(None)
    span_ms = sum(spans)
    rows = []
    for name, t in table.items():
        if not t["launches"]:
            continue
        secs = t["ms"] / 1e3
        t_hbm = t["bytes"] / (hbm_gbs * 1e9)
        t_int = sum(t[k] / peaks[k] for k in peaks)
        bound = "hbm" if t_hbm >= t_int else "integer"
        rows.append({"kernel": name, "launches": t["launches"] // steps,
                     "us_per_proof": 1e3 * t["ms"] / steps,
                     "avg_launch_us": 1e3 * t["ms"] / t["launches"],
                     "share_of_device_span": t["ms"] / span_ms, "bound": bound,
                     "frac": max(t_hbm, t_int) / secs if secs > 0 else None,
                     "bytes_per_launch": t["bytes"] / t["launches"],
                     "products_per_launch": sum(t[k] for k in peaks) / t["launches"]})
    rows.sort(key=lambda r: -r["share_of_device_span"])
    top = rows[0]
    t = table[top["kernel"]]
    secs = t["ms"] / 1e3
    prods = sum(t[k] for k in peaks)
    if top["bound"] == "hbm":
        achieved, peak, unit = t["bytes"] / secs / 1e9, hbm_gbs, "GB/s"
        peak_source = f"hbm_gbs, {pk_kind}"
    else:
        # the ceiling of this kernel's product mix at the measured throughputs
        t_int = sum(t[k] / peaks[k] for k in peaks)
        achieved, peak, unit = prods / secs / 1e9, prods / t_int / 1e9, "Gproducts/s"
        peak_source = ("measured GF(2^128) product throughput of this GPU (bitz_diag_gf_peak: "
                       + ", ".join(f"{k} {v / 1e9:.1f} G/s" for k, v in peaks.items())
                       + "), weighted by the kernel's product mix")
    traffic = profile_figure(top["kernel"], "traffic_bytes_per_launch", tag)
    return {"kernel": top["kernel"], "bound": top["bound"], "achieved": achieved, "peak": peak,
            "unit": unit, "frac": achieved / peak, "peak_source": peak_source,
            "traffic": traffic,
            "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum, mean over the "
                               f"captured launches of the committed summary "
                               f"profiles/{top['kernel']}_{tag}.md") if traffic else None,
            "algorithmic_bytes_per_launch": top["bytes_per_launch"],
            "products_per_launch": top["products_per_launch"],
            "launches_per_proof": top["launches"], "avg_launch_us": top["avg_launch_us"],
            "share_of_device_span": top["share_of_device_span"],
            "share_of_kernel_time_ncu": profile_figure(
                "launches", f"{top['kernel']}_share_of_kernel_time", tag),
            "share_note": "share_of_device_span: this run's CUDA-event kernel time over the proofs' "
                          "device span (host waits included); share_of_kernel_time_ncu: the "
                          "committed ncu launch list's share of summed kernel time",
            "mode": "every sumcheck round its own launch (as under ncu), events per launch",
            "kernels": rows[:8]}


def replica_value(world, blocks, steps, slowest_ms):
    """Whole-job blocks/s of `world` replicas, each proving `steps` proofs of
    `blocks` blocks: every rank's blocks over the slowest rank's time."""
    return world * blocks * steps / (slowest_ms / 1000.0)


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
    """256 sha256-block-aligned proofs, k ~ U{0..32} (seed 3), concurrent on
    ``args.lanes`` lanes, against the same 256 proved one after another by the
    plain single-proof call on the default lane (CircuitProofSystem.prove) and
    on one pool lane."""
    from bitz_b200 import statements
    mix = statements.batch_mix(3, 256, 32)
    systems = [bz.CircuitProofSystem(kind, inp, out, args.security) for kind, inp, out in mix]
    blocks = sum(statements.blocks_proven(kind, inp.size) for kind, inp, _ in mix)
    # warm-up: every lane's scratch grows to the largest shape of the mix
    largest = sorted(range(len(mix)), key=lambda i: -mix[i][1].size)[:args.lanes]
    bz.batch_prove([systems[i] for i in largest], args.lanes)
    bz.batch_prove([systems[largest[0]]], 1)
    systems[largest[0]].prove()
    bz.batch_prove(systems, args.lanes)
    res = {}
    # the plain path: one proof after another through the single-proof call
    bz.l2_flush()
    plain, lat = [], []
    t0 = time.perf_counter()
    for ps in systems:
        t = time.perf_counter()
        plain.append(ps.prove()[0])
        lat.append(1e3 * (time.perf_counter() - t))
    res["plain"] = (blocks / (time.perf_counter() - t0), lat, plain)
    for name, lanes in (("pool_lane", 1), ("batched", args.lanes)):
        bz.l2_flush()
        g0 = bz.gate_stats()
        t0 = time.perf_counter()
        proofs, lat = bz.batch_prove(systems, lanes)
        wall = time.perf_counter() - t0
        res[name] = (blocks / wall, lat, proofs, gate_delta(g0, bz.gate_stats()))
    same = res["plain"][2] == res["batched"][2] == res["pool_lane"][2]
    return {"workload": "256 x sha256-block-aligned, k ~ U{0..32} blocks (SplitMix64 seed 3), "
                        f"pcs-security-bits {args.security}",
            "blocks": blocks, "lanes": args.lanes,
            "value": res["batched"][0], "unit": "blocks/s",
            "sequential_plain_value": res["plain"][0],
            "speedup_vs_sequential_plain": res["batched"][0] / res["plain"][0],
            "sequential_pool_lane_value": res["pool_lane"][0],
            "latency_ms": {"p50": pct(res["batched"][1], 0.5), "p99": pct(res["batched"][1], 0.99)},
            "sequential_plain_latency_ms": {"p50": pct(res["plain"][1], 0.5),
                                            "p99": pct(res["plain"][1], 0.99)},
            "proofs_identical_to_alone": same,
            "gate": res["batched"][3]}


def gate_delta(g0, g1):
    """Device-gate activity between two gate_stats() readings: allocations
    (scratch growth) and the seconds allocations and resident stretches
    waited for each other."""
    return {"allocs": g1["allocs"] - g0["allocs"],
            "alloc_wait_s": round(g1["alloc_wait_s"] - g0["alloc_wait_s"], 6),
            "resident_wait_s": round(g1["resident_wait_s"] - g0["resident_wait_s"], 6)}


def large(args, bz, steps=5, warmup=2):
    """sha256-chain n=1024 (64 KiB, SplitMix64 seed 2) at PCS security 128 (unique
    decoding, no OOD): one proof per step, device time by CUDA events on the
    prover's stream, L2 flushed before each; then the roofline of its dominant
    kernel, as for the main workload."""
    from bitz_b200 import statements
    inp, out, _ = statements.instance("sha256-chain", 1024, 2)
    ps = bz.CircuitProofSystem("sha256-chain", inp, out, 128)
    for _ in range(warmup):
        ps.prove(restage=False)
    spans, e2e = [], []
    for _ in range(steps):
        bz.l2_flush()
        _, t = ps.prove(restage=False)
        spans.append(t["device_ms"])
    for _ in range(steps):
        bz.l2_flush()
        t0 = time.perf_counter()
        ps.prove(restage=True)
        e2e.append(1e3 * (time.perf_counter() - t0))
    pk, pk_kind = peaks()
    roof = roofline(bz, ps, 2, pk["hbm_gbs"], pk_kind, tag="sha256-chain-n1024")
    return {"workload": "sha256-chain n=1024 pcs-security-bits 128 (seed 2)", "blocks": 1024,
            "roofline": roof,
            "steps": steps, "value": 1024 * steps / (sum(spans) / 1e3), "unit": "blocks/s",
            "latency_ms": {"p50": statistics.median(spans), "p99": pct(spans, 0.99)},
            "e2e": {"value": 1024 * steps / (sum(e2e) / 1e3), "unit": "blocks/s",
                    "latency_ms": {"p50": statistics.median(e2e), "p99": pct(e2e, 0.99)}}}


def serve_sweep(args, bz, requests, max_rates, emit=False):
    """Open-loop Poisson arrivals into the prove server, the rate swept upward
    by 1.5x until p99 latency exceeds 10x the single-request p99 (or after
    ``max_rates`` rates). Returns the sweep and the plain arm: the same stream
    proved one request after another through the single-proof call
    (statement preparation included, as a served request's latency includes
    it)."""
    from bitz_b200 import statements
    mix = statements.serve_mix(4, requests, 512)
    blocks = [statements.blocks_proven(k, i.size) for k, i, _ in mix]
    # circuit shapes are built once per (circuit, size) and cached, as the
    # reference's benchmark excludes setup: build every shape of the stream
    t0 = time.perf_counter()
    shapes = {}
    for kind, inp, out in mix:
        shapes.setdefault((kind, inp.size), (kind, inp, out))
    for kind, inp, out in shapes.values():
        bz.CircuitProofSystem(kind, inp, out, args.security).prove()
    setup_s = time.perf_counter() - t0
    # the plain arm: each request prepared and proved alone, one after another
    alone, plain_lat = [], []
    t0 = time.perf_counter()
    for kind, inp, out in mix:
        t = time.perf_counter()
        alone.append(bz.CircuitProofSystem(kind, inp, out, args.security).prove()[0])
        plain_lat.append(1e3 * (time.perf_counter() - t))
    plain_bps = sum(blocks) / (time.perf_counter() - t0)
    rng = random.Random(4)
    sweep = []
    with bz.ProveServer(lanes=args.lanes, hbm_budget=96 << 30, security_bits=args.security) as srv:
        # warm-up: every lane's scratch grows to the largest shape of the stream
        big = max(mix, key=lambda m: m[1].size)
        warm = [srv.submit(*big) for _ in range(args.lanes)]
        for t in warm:
            while srv.poll(t, 50) is None:
                pass
        # single-request latency: each request alone on an idle server, submit
        # to proof bytes (statement preparation included)
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
        for _ in range(max_rates):
            gaps = [rng.expovariate(rate) for _ in mix]
            g0 = bz.gate_stats()
            tickets, t0 = [], time.perf_counter()
            due = t0
            for (kind, inp, out), g in zip(mix, gaps):
                due += g
                while time.perf_counter() < due:
                    time.sleep(min(0.0005, max(0.0, due - time.perf_counter())))
                tickets.append(srv.submit(kind, inp, out))
            got = {}
            while len(got) < len(tickets):
                for t in tickets:
                    if t not in got:
                        r = srv.poll(t, 2)
                        if r is not None:
                            got[t] = r
            wall = time.perf_counter() - t0
            lat = [got[t][1] for t in tickets]
            same = all(got[t][0] == a for t, a in zip(tickets, alone))
            p99 = pct(lat, 0.99)
            point = {"rate_rps": rate, "value": sum(blocks) / wall, "unit": "blocks/s",
                     "latency_ms": {"p50": pct(lat, 0.5), "p99": p99},
                     "peak_in_flight": srv.stats()["peak_in_flight"],
                     "gate": gate_delta(g0, bz.gate_stats()),
                     "proofs_identical_to_alone": same}
            sweep.append(point)
            if emit:
                print(json.dumps(dict(point, metric="SHA-256 blocks proven/sec (serving)",
                                      single_request_latency_ms={"p50": pct(alone_served, 0.5),
                                                                 "p99": single},
                                      lanes=args.lanes, requests=len(mix))), flush=True)
            if p99 > 10 * single or rate > 2000:
                break
            rate *= 1.5
    below = [pt for pt in sweep if pt["latency_ms"]["p99"] <= 10 * single]
    best = max(below or sweep[:1], key=lambda pt: pt["value"])
    return {"workload": "Poisson arrivals; 50% sha256-2kb, 50% sha256-block-aligned "
                        "k = floor(2^U(0,9)) in 1..512 (seed 4)",
            "requests": len(mix), "blocks": sum(blocks), "lanes": args.lanes,
            "rate_rps": best["rate_rps"], "value": best["value"], "unit": "blocks/s",
            "latency_ms": best["latency_ms"], "gate": best["gate"],
            "single_request_latency_ms": {"p50": pct(alone_served, 0.5), "p99": single},
            "plain_sequential_value": plain_bps,
            "speedup_vs_plain_sequential": best["value"] / plain_bps,
            "plain_latency_ms": {"p50": pct(plain_lat, 0.5), "p99": pct(plain_lat, 0.99)},
            "proofs_identical_to_alone": all(pt["proofs_identical_to_alone"] for pt in sweep),
            "rates_swept": len(sweep), "shapes_prebuilt": len(shapes), "setup_s": setup_s,
            "note": "the point reported is the highest-throughput rate whose p99 stays within "
                    "10x the single-request p99"}


def serve(args):
    """``--serve``: the full serving sweep, one JSON line per rate, then the summary."""
    import bitz_b200 as bz
    bz.set_device(dist_env()[2])
    resolve_lanes(args, bz)
    summary = serve_sweep(args, bz, args.serve_requests, 30, emit=True)
    print(json.dumps(dict(summary, metric="SHA-256 blocks proven/sec (serving)")))


def ours(args):
    world, rank, local = dist_env()
    import bitz_b200 as bz
    lib_path = os.path.join(ROOT, "bitz_b200", "libbitz_b200.so")
    if not os.path.exists(lib_path):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "bitz_b200")], check=True)
    dist = Dist(world)
    bz.set_device(local)
    resolve_lanes(args, bz)
    inputs, outputs, _ = statement(args)
    blocks = blocks_proven(args, inputs.size)
    ps = bz.CircuitProofSystem(args.circuit, inputs, outputs, args.security)
    for _ in range(args.warmup):
        ps.prove(restage=False)
    # device-resident timed region: the statement stays staged, the L2 is
    # flushed before every proof, each proof timed by CUDA events on its stream
    dist.barrier()
    launches0 = bz.launch_count()
    wait0 = bz.round_wait_stats()
    with Clocks(local) as clk:
        spans, host_ms = [], []
        for _ in range(args.steps):
            bz.l2_flush()
            proof, times = ps.prove(restage=False)
            spans.append(times["device_ms"])
            host_ms.append(times["witness_ms"] + times["commit_ms"] + times["prove_ms"])
    launches = bz.launch_count() - launches0
    wait1 = bz.round_wait_stats()
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
    value = replica_value(world, blocks, args.steps, dev_total_ms)
    e2e = world * blocks * args.steps / e2e_s
    stats = ps.stats()
    h2d = 4 * (8 + 16) * stats["compressions"] + 8 * stats["compressions"] + (inputs.size + 7) // 8 \
        + inputs.size + 256
    pk, pk_kind = peaks()
    roof = roofline(bz, ps, 3, pk["hbm_gbs"], pk_kind)
    batch = big = serving = None
    if world == 1 and not args.no_batch:
        batch = batched(args, bz)
    if world == 1 and not args.no_large:
        big = large(args, bz)
    if world == 1 and not args.no_serving:
        serving = serve_sweep(args, bz, args.serving_requests, args.serving_rates)
    line = None
    if rank == 0:
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
            "round_split": {
                "rounds_per_proof": (wait1[1] - wait0[1]) / args.steps,
                "host_waiting_ms_per_proof": 1e3 * (wait1[0] - wait0[0]) / args.steps,
                "host_ms_per_proof": statistics.mean(host_ms),
                "note": "host_waiting: the prover's host thread waiting for round results "
                        "(device work plus the PCIe round trip); the rest of host_ms is the host's "
                        "own transcript work (Keccak absorbs, challenges, grinding)"},
            "roofline": roof,
            "clocks": clk.summary(),
            "proof_bytes": len(proof),
            "peaks": pk_kind,
        }
        if batch:
            line["batched"] = batch
        if big:
            line["large"] = big
        if serving:
            line["serving"] = serving
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args, inputs, outputs, blocks)
        print(json.dumps(line))
    dist.close()


def resolve_lanes(args, bz):
    if args.lanes is None:
        args.lanes = int(bz.TUNING.get("lanes", 16))


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
