#!/usr/bin/env python
"""Benchmark of the B200 bit-plane traverser (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

A step is one pass of the hot path over one batch: the headline workload
advances a 65536 x 65536 Game of Life grid (bit planes, 512 MiB packed,
Bernoulli(0.35) seeded input) by 1000 generations.  Under torchrun the grid
is 65536 wide and N*65536 tall, split into one 65536-row band per rank, with
a halo exchange of K rows each way between neighbouring ranks (NCCL) before
every K-generation pass: weak scaling.

value     Gcell-updates/s over all ranks, device-timed (CUDA events on the
          launching stream), inputs resident in HBM, max over ranks.
e2e       the same metric through the C-ABI with host buffers: every step
          uploads the bit-plane image from pinned host memory, runs, and
          downloads the result.
roofline  the strip kernel against the measured integer-logic peak (the
          binding roof for k >= 2) and against the measured HBM copy peak.
cpu_baseline  Cellato's own CPU traverser (oracle/_ref, compiled from the
          reference headers) on the host cores, on a bounded sample.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "gol-65536": dict(automaton=0, x=65536, y=65536, gens=1000, probs=[0.65, 0.35], seed=42,
                      desc="game-of-life 65536x65536 bit_planes, Bernoulli(0.35), 1000 generations per step"),
    "wire-32768": dict(automaton=1, x=32768, y=32768, gens=2000, probs=[0.60, 0.05, 0.05, 0.30], seed=42,
                       desc="wire 32768x32768 bit_planes (2 planes), categorical "
                            "(empty .60, head .05, tail .05, conductor .30), 2000 generations per step"),
    "excitable-32768": dict(automaton=2, x=32768, y=32768, gens=2000, probs=[0.125] * 8, seed=42,
                            desc="excitable (Greenberg-Hastings, 8 states) 32768x32768 bit_planes (3 planes), "
                                 "uniform states, 2000 generations per step"),
    "gol-1024": dict(automaton=0, x=1024, y=1024, gens=100, probs=[0.5, 0.5], seed=42,
                     desc="game-of-life 1024x1024, Bernoulli(0.5), 100 generations per step"),
}
METRIC = "Gcell-updates/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.json")
FALLBACK_HBM_GBS = 6650.0

CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---- clocks -----------------------------------------------------------------------------------

class ClockSampler:
    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(prefix="cb2_clocks_", suffix=".csv")
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={CLOCK_QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v for v in vis.split(",") if v.strip()]
        if local_rank < len(ids) and ids[local_rank].strip().isdigit():
            return int(ids[local_rank])
    return local_rank


# ---- CPU baseline: Cellato's own CPU traverser ------------------------------------------------

def cpu_sample(automaton: int, probs, target_s: float, threads: int | None = None) -> dict:
    """Times the reference CPU simple traverser (bit_planes, 64-bit words) with
    one independent grid per host thread on a 4096x4096 sample."""
    from oracle import oracle as O

    threads = threads or os.cpu_count() or 1
    x = y = 4096
    cells = O.init_cells(x, y, 1, O.thresholds(probs))
    if O.ref_available():
        kind = "reference"
        run = lambda gens: O.ref_bench(automaton, cells, gens, threads, "bit_planes", 64)  # noqa: E731
    else:  # the C restatement, single-threaded
        kind, threads = "port", 1
        planes = O.pack("bit_planes", cells, O.PLANES[automaton], 32).view("uint32")

        def run(gens):
            t0 = time.perf_counter()
            O.run_bit_planes(automaton, planes, x, y, gens)
            return time.perf_counter() - t0
    probe = max(run(2), 1e-4)
    gens = max(2, int(target_s / probe * 2))
    secs = run(gens)
    value = threads * x * y * gens / secs / 1e9
    return {"value": value, "unit": METRIC, "cores": threads, "kind": kind,
            "sample": f"{threads} host thread(s), each its own {x}x{y} grid, {gens} generations, "
                      f"Cellato CPU simple traverser, bit_planes layout, 64-bit words ({secs:.2f} s)"}


def reference_arm(args, wl) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    target = 8.0
    samples = []
    for _ in range(args.warmup):
        cpu_sample(wl["automaton"], wl["probs"], 1.0)
    for _ in range(args.steps):
        samples.append(cpu_sample(wl["automaton"], wl["probs"], target))
    value = statistics.mean(s["value"] for s in samples)
    base = dict(samples[-1])
    base["value"] = value
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
           "config": {"workload": wl["desc"], "sample": base["sample"]},
           "cpu_baseline": base, "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---- the B200 arm ------------------------------------------------------------------------------

def measured_peaks() -> dict:
    try:
        with open(PEAKS_FILE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def traffic_for(kernel_key: str):
    try:
        with open(TRAFFIC_FILE) as f:
            t = json.load(f)
        return t.get(kernel_key)
    except (OSError, ValueError):
        return None


BATCH_PROBS = {0: [0.65, 0.35], 1: [0.60, 0.05, 0.05, 0.30], 2: [0.125] * 8}


# The lowered DSL automata of the batched DSL line: every bundled automaton
# without a hand-written network and the two stochastic examples.
BATCH_DSL = ["brian", "critters", "cyclic", "forest-fire", "fluid", "maze", "traffic", "lightning-forest",
             "noisy-life"]


def batch_workload(n: int, seed: int = 2024, automata=(0, 1, 2)):
    """n independent grids: sides log-uniform in [64, 4096] (widths rounded to
    multiples of 32), automaton uniform over `automata`, steps log-uniform in
    [10, 1000]."""
    import numpy as np

    rng = np.random.default_rng(seed)
    lo, hi = math.log(64), math.log(4096)
    specs = []
    for i in range(n):
        x = int(min(4096, max(64, 32 * round(math.exp(rng.uniform(lo, hi)) / 32))))
        y = int(min(4096, max(64, round(math.exp(rng.uniform(lo, hi))))))
        a = automata[int(rng.integers(0, len(automata)))]
        steps = int(round(math.exp(rng.uniform(math.log(10), math.log(1000)))))
        specs.append((a, x, y, steps))
    return specs


def batch_probs(cb, a):
    if a in BATCH_PROBS:
        return BATCH_PROBS[a]
    states = cb.automaton_info(a)[2]
    return [0.5, 0.25, 0.25] if states == 3 else [1.0 / states] * states  # exact binary fractions


def bench_batch(cb, torch, stream, n: int, runs: int, automata=(0, 1, 2)) -> dict:
    specs = batch_workload(n, automata=automata)
    grids = []
    for i, (a, x, y, _) in enumerate(specs):
        g = cb.DeviceGrid(a, x, y)
        g.fill_random(1000 + i, batch_probs(cb, a), stream=stream)
        g.set_seed(5000 + i)
        grids.append(g)
    steps = [s for (_, _, _, s) in specs]
    batch = cb.Batch(grids, steps)
    info = batch.info()
    for _ in range(2):
        batch.run(stream)
    batch.wait(stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(runs):
        batch.run(stream)
    e1.record(stream)
    batch.wait(stream)
    ms = e0.elapsed_time(e1) / runs
    batch.run_per_grid(stream)  # warm-up of the per-grid plans
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    batch.run_per_grid(stream)
    f1.record(stream)
    f1.synchronize()
    per_ms = f0.elapsed_time(f1)
    batch.close()
    for g in grids:
        g.close()
    cells = info["cell_updates"]
    names = ", ".join(cb.automaton_info(a)[0] if isinstance(a, int) else a for a in automata)
    return {"workload": f"{n} grids, sides log-uniform [64,4096] (widths multiple of 32), automaton uniform "
                        f"{{{names}}}, steps log-uniform [10,1000], seeded inits",
            "value": cells / (ms * 1e-3) / 1e9, "unit": METRIC, "ms_per_run": ms, "runs": runs,
            "cell_updates_per_run": cells, "tasks": info["tasks"], "persistent_ctas": info["persistent_ctas"],
            "per_grid_value": cells / (per_ms * 1e-3) / 1e9, "per_grid_ms_per_run": per_ms,
            "speedup_vs_per_grid": per_ms / ms,
            "path": "cb2_batch_run (persistent tile-queue kernel, CUDA graph replay) vs cb2_batch_run_per_grid "
                    "(cb2_grid_run per grid)"}


def serve_workload(n: int, seed: int = 7, automata=(0, 1, 2)):
    """Requests: sides log-uniform in [128, 16384] (widths multiples of 32),
    steps log-uniform in [1, 10000], automaton uniform over `automata`, seeded inputs."""
    import numpy as np

    rng = np.random.default_rng(seed)
    lo, hi = math.log(128), math.log(16384)
    out = []
    for i in range(n):
        x = int(min(16384, max(128, 32 * round(math.exp(rng.uniform(lo, hi)) / 32))))
        y = int(min(16384, max(128, round(math.exp(rng.uniform(lo, hi))))))
        steps = int(max(1, round(math.exp(rng.uniform(0.0, math.log(10000))))))
        out.append((automata[int(rng.integers(0, len(automata)))], x, y, steps, 5000 + i))
    return out


def serve_stream(cb, specs, rate: float, per_request: bool, seed: int = 11, **server_opts) -> dict:
    """Submits `specs` with Poisson arrivals at `rate` req/s; returns latency
    percentiles (submit to result) and throughput over the makespan."""
    import numpy as np

    gaps = np.random.default_rng(seed).exponential(1.0 / rate, len(specs))
    with cb.Server(per_request=per_request, **server_opts) as srv:
        t0 = time.perf_counter()
        due = 0.0
        ids = []
        for (a, x, y, steps, sd), gap in zip(specs, gaps):
            due += gap
            while time.perf_counter() - t0 < due:
                time.sleep(min(0.0005, max(0.0, due - (time.perf_counter() - t0))))
            ids.append(srv.submit(a, x, y, steps, sd, batch_probs(cb, a)))
        srv.drain(1200)
        st = [srv.status(i) for i in ids]
        stats = srv.stats()
    lat = np.array([r["done_s"] - r["submit_s"] for r in st])
    span = max(r["done_s"] for r in st) - min(r["submit_s"] for r in st)
    cells = sum(x * y * steps for (_, x, y, steps, _) in specs)
    return {"rate_req_s": rate, "requests": len(specs), "failed": sum(r["state"] != "done" for r in st),
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "throughput": cells / span / 1e9, "makespan_s": span, "rounds": stats["rounds"],
            "server_plan_s": stats["plan_s"], "server_wait_s": stats["wait_s"], "batch_tasks": stats["tasks"]}


def bench_serve(cb, n: int, rates, automata=(0, 1, 2)) -> dict:
    specs = serve_workload(n, automata=automata)
    serve_stream(cb, specs[:20], 1000.0, False)  # warm-up: graph capture, pools
    serve_stream(cb, specs[:20], 1000.0, True)
    points = []
    for rate in rates:
        # the median of three runs of the batched server (one Poisson stream each; the
        # makespan is a few tenths of a second, so single runs vary by 10-20 %)
        runs = sorted((serve_stream(cb, specs, rate, False) for _ in range(3)), key=lambda r: r["throughput"])
        batched = dict(runs[1], throughput_of_runs=[r["throughput"] for r in runs])
        plain = serve_stream(cb, specs, rate, True)
        points.append({"rate_req_s": rate, "batched": batched, "per_request": plain,
                       "throughput_ratio": batched["throughput"] / plain["throughput"]})
    names = ", ".join(cb.automaton_info(a)[0] if isinstance(a, int) else a for a in automata)
    return {"workload": f"{n} requests per rate, Poisson arrivals, sides log-uniform [128,16384] (widths multiple "
                        f"of 32), steps log-uniform [1,10000], automaton uniform {{{names}}}, seeded inits",
            "unit": METRIC, "latency": "submit to finished (checksum ready), ms",
            "memory_budget": "min(150 GiB, 80% of free device memory) of bit-plane state",
            "path": "cb2_server (continuous batching, persistent batch kernel per round) vs cb2_server per_request=1 "
                    "(one request at a time, one launch sequence each)",
            "points": points}


def launches_per_run(gens: int, k: int) -> int:
    n, left = 0, gens
    while left > 0:
        step = k
        while step > left:
            step //= 2
        left -= step
        n += 1
    return n


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="gol-65536", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="run the library's default plan instead of timing candidates first (for profiler runs, "
                         "whose serialised launches distort the candidates' timings)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--serve-dsl-requests", type=int, default=300,
                    help="requests of the served point over the lowered DSL automata (0 = skip)")
    ap.add_argument("--batch-grids", type=int, default=4096)
    ap.add_argument("--batch-dsl-grids", type=int, default=1024,
                    help="grids of the batched line over the lowered DSL automata (0 = skip)")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return reference_arm(args, wl)
    if args.warmup < 3:
        raise SystemExit("--warmup must be at least 3")

    import torch
    import torch.distributed as dist

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    import cellato_b200 as cb

    a, x, y, gens = wl["automaton"], wl["x"], wl["y"], wl["gens"]
    name, P, _ = cb.automaton_info(a)
    cells = x * y
    stream = torch.cuda.current_stream()
    tuned = None if args.no_autotune else cb.autotune(a, x, y, budget_ms=4000)
    plan = cb.plan(a, x, y)
    k = plan["temporal_steps"]
    if world == 1:
        grid = cb.DeviceGrid(a, x, y)
        grid.fill_random(wl["seed"], wl["probs"], stream=stream)
    else:
        # one grid of world*y rows split into bands, one per rank (NCCL halo exchange per pass)
        from cellato_b200.bands import BandGrid

        grid = BandGrid(a, x, y * world, rank, world)
        grid.fill_random(wl["seed"], wl["probs"], stream=stream)
        # every rank must take the same passes (one halo exchange each): use rank 0's depth
        kt = torch.tensor([grid.plan_k()], dtype=torch.int64, device="cuda")
        dist.broadcast(kt, 0)
        k = int(kt.item())

    run_kw = {} if world == 1 else {"temporal_steps": k}

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident timing ----
    for _ in range(args.warmup):
        grid.run(gens, **run_kw, stream=stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_index(local_rank)) if local_rank == 0 else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        grid.run(gens, **run_kw, stream=stream)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop() if sampler else None
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = world * cells * gens * args.steps / (ms * 1e-3) / 1e9
    launches = launches_per_run(gens, k) * args.steps

    # ---- roofline of the strip kernel ----
    avg_launch_s = ms * 1e-3 / launches
    gens_per_launch = gens * args.steps / launches
    bytes_per_launch = 2 * P * cells / 8  # read + write every plane once
    hbm_gbs = bytes_per_launch / avg_launch_s / 1e9
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs", FALLBACK_HBM_GBS)
    lop3_peak = cb.measure_lop3_peak()
    alu_per_word, shfl_per_word = cb.network_ops(a)
    int_ops_per_launch = alu_per_word * (cells / 32) * gens_per_launch
    int_gops = int_ops_per_launch / avg_launch_s / 1e9
    int_frac = int_gops / (lop3_peak / 1e9)
    hbm_frac = hbm_gbs / hbm_peak
    kernel_key = (f"pipe_kernel<{name},K={k},V={plan['words_per_lane']},L={plan['levels_per_warp']},"
                  f"R={plan['rows_per_step']}>@{x}x{y}")
    traffic = traffic_for(kernel_key)
    roof = {
        "bound": "int" if int_frac >= hbm_frac else "hbm",
        "kernel": kernel_key,
        "achieved": int_gops if int_frac >= hbm_frac else hbm_gbs,
        "peak": lop3_peak / 1e9 if int_frac >= hbm_frac else hbm_peak,
        "unit": "Gop/s" if int_frac >= hbm_frac else "GB/s",
        "frac": max(int_frac, hbm_frac),
        "traffic": traffic,
        "peak_source": ("measured LOP3 issue rate (cb2_measure_lop3_peak, this run)" if int_frac >= hbm_frac else
                        ("measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6.65 TB/s")),
        "int": {"achieved_gops": int_gops, "peak_gops": lop3_peak / 1e9, "frac": int_frac,
                "ops_per_word_per_generation": alu_per_word, "shuffles_per_word_per_generation": shfl_per_word},
        "hbm": {"achieved_gbs": hbm_gbs, "peak_gbs": hbm_peak, "frac": hbm_frac,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "avg_launch_ms": avg_launch_s * 1e3,
        "generations_per_launch": gens_per_launch,
    }

    # ---- end to end through the public API with host buffers ----
    nbytes = cb.layout_bytes(a, "bit_planes", 64, x, y)
    host_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    host_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    if world == 1:
        grid.download("bit_planes", 64, stream=stream, out=host_in.numpy())
        host_img = cb.HostGrid(a, "bit_planes", 64, x, y, host_in.numpy())

        def e2e_step():
            grid.upload(host_img, stream=stream)
            grid.run(gens, **run_kw, stream=stream)
            grid.download("bit_planes", 64, stream=stream, out=host_out.numpy())
    else:
        g0, nb = grid.ghost, grid.band
        band_in = host_in.view(torch.int32).view(P, nb, x // 32)
        band_out = host_out.view(torch.int32).view(P, nb, x // 32)
        band_in.copy_(grid.planes[:, g0:g0 + nb])

        def e2e_step():
            grid.planes[:, g0:g0 + nb].copy_(band_in, non_blocking=True)
            grid.run(gens, **run_kw, stream=stream)
            band_out.copy_(grid.planes[:, g0:g0 + nb], non_blocking=True)
            torch.cuda.current_stream().synchronize()
    e2e_step()
    torch.cuda.synchronize()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    f0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    f1.record(stream)
    f1.synchronize()
    wall = time.perf_counter() - w0
    barrier()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1))
    e2e_wall = max_over_ranks(wall)
    e2e_value = world * cells * gens * args.steps / (e2e_ms * 1e-3) / 1e9

    if world == 1:
        grid.close()
    else:
        del grid
    torch.cuda.synchronize()
    batched = None
    if not args.no_batch:
        batched = bench_batch(cb, torch, stream, args.batch_grids, max(3, args.steps))
    batched_dsl = None
    if not args.no_batch and args.batch_dsl_grids > 0 and all(n in cb.AUTOMATA for n in BATCH_DSL):
        batched_dsl = bench_batch(cb, torch, stream, args.batch_dsl_grids, 3, automata=BATCH_DSL)
    served = None
    if not args.no_serve:
        served = bench_serve(cb, args.serve_requests, [100.0, 1000.0, 5000.0, 20000.0])
    served_dsl = None
    if not args.no_serve and args.serve_dsl_requests > 0 and all(n in cb.AUTOMATA for n in BATCH_DSL):
        served_dsl = bench_serve(cb, args.serve_dsl_requests, [5000.0], automata=BATCH_DSL)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(a, wl["probs"], args.cpu_seconds)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": wl["desc"], "automaton": name, "x_size": x, "y_size": y,
                   "generations_per_step": gens, "plan": plan, "autotuned": tuned,
                   "l2": (f"inputs larger than L2: each of the {P} plane(s) of each buffer is "
                          f"{x * y // 8 // 2**20} MiB at {x}x{y}; a K-generation pass streams all of them"),
                   "parallelism": (f"row bands x{world}: one {x}x{y * world} grid, {y} rows per GPU, NCCL halo "
                                   f"exchange of K rows each way per pass" if world > 1 else "single GPU")},
        "roofline": roof,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                "wall_s": e2e_wall,
                "path": ("cb2_grid_upload(bit_planes) + cb2_grid_run + cb2_grid_download, pinned host buffers"
                         if world == 1 else "band planes from pinned host memory + BandGrid.run (halo exchange + "
                                            "cb2_band_pass per pass) + band planes back, per rank")},
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "batched": batched,
        "batched_dsl": batched_dsl,
        "served": served,
        "served_dsl": served_dsl,
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
