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
          downloads the result into pinned host memory; on one GPU the
          steps are pipelined over two device grids and two copy streams
          (cb2_grid_upload_async / cb2_grid_download_async), so copies of
          neighbouring steps overlap a step's run.
roofline  the strip kernel against the measured integer-logic peak (the
          binding roof for k >= 2) and against the measured HBM copy peak.
cpu_baseline  Cellato's own CPU traverser (oracle/_ref, compiled from the
          reference headers) on the benchmark grid itself, on the host cores:
          all threads (each on a band of the grid's rows) and one thread (the
          whole grid), over a timed sub-range of the step's generations, in
          its fastest layout (bit_planes, 64-bit words); and one thread in the
          standard layout on a 64-row band of the grid.
workloads  (one GPU) the WireWorld and Greenberg-Hastings 32768^2 x 2000
          workloads, each with its own roofline, e2e and clocks.
temporal_depths  (one GPU) the headline at k = 1, 2, 4, 8 generations per
          HBM round trip, each with its fastest kernel, beside the autotuned k.
layouts   (one GPU) the headline step through the bit_planes, bit_array and
          tiled_bit_planes host layouts (conversions on the device at the
          boundary), with the boundary's share of each step.
batched, served, batched_dsl, served_dsl  many grids in one persistent kernel,
          and continuous-batching serving, each against one grid at a time.

--impl reference times Cellato's CPU traverser on the same grid on all host
threads (each step a timed sub-range of the step's generations) and prints
the same metric for the same config.
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
    "gol-65536": dict(automaton=0, name="game-of-life", planes=1, x=65536, y=65536, gens=1000, probs=[0.65, 0.35], seed=42,
                      desc="game-of-life 65536x65536 bit_planes, Bernoulli(0.35), 1000 generations per step"),
    "wire-32768": dict(automaton=1, name="wire", planes=2, x=32768, y=32768, gens=2000, probs=[0.60, 0.05, 0.05, 0.30], seed=42,
                       desc="wire 32768x32768 bit_planes (2 planes), categorical "
                            "(empty .60, head .05, tail .05, conductor .30), 2000 generations per step"),
    "excitable-32768": dict(automaton=2, name="excitable", planes=3, x=32768, y=32768, gens=2000, probs=[0.125] * 8, seed=42,
                            desc="excitable (Greenberg-Hastings, 8 states) 32768x32768 bit_planes (3 planes), "
                                 "uniform states, 2000 generations per step"),
    "gol-1024": dict(automaton=0, name="game-of-life", planes=1, x=1024, y=1024, gens=100, probs=[0.5, 0.5], seed=42,
                     desc="game-of-life 1024x1024, Bernoulli(0.5), 100 generations per step"),
}
METRIC = "Gcell-updates/s"
# Logic ops per word and generation that a rule's network adds when a plan
# pushes one row per step, beyond cb2_network_ops (which counts the pair
# evaluation of two or more rows per step): game-of-life 10 instead of 9,
# wire 10 instead of 8.
ROW_BY_ROW_EXTRA_OPS = {0: 1, 1: 2}
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

def headline_config(wl, world: int) -> dict:
    """The workload description both arms report (so the lines compare like for like)."""
    x, y = wl["x"], wl["y"]
    P = wl["planes"]
    return {"workload": wl["desc"] + (f"; {world} row bands of {y} rows (one {x}x{y * world} grid)"
                                      if world > 1 else ""),
            "automaton": wl["name"], "x_size": x, "y_size": y * world, "generations_per_step": wl["gens"],
            "seed": wl["seed"], "state_probabilities": wl["probs"],
            "l2": (f"inputs larger than L2: each of the {P} plane(s) of each buffer is {x * y // 8 // 2**20} MiB "
                   f"per GPU; every K-generation pass streams all of them"),
            "parallelism": (f"row bands x{world}, NCCL halo exchange of K rows each way per pass" if world > 1
                            else "single GPU")}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_threads(rows: int) -> int:
    """Host threads for the CPU samples: all cores, rounded down to a divisor of the rows."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    return max(t for t in range(1, n + 1) if rows % t == 0)


class ReferenceSample:
    """Cellato's own CPU simple traverser (bit_planes layout, 64-bit words;
    oracle/_ref, compiled from the reference headers) on the benchmark's grid
    itself: the seeded input built as bit planes, then advanced (a) by all
    host threads, each on its band of rows of the grid as a torus of its own,
    so that every cell of the grid advances once per generation, and (b) by
    one thread over the whole grid.  Without the reference build, the oracle's
    C restatement (single-threaded, whole grid) stands in."""

    def __init__(self, wl, world: int):
        from oracle import oracle as O

        self.O = O
        self.a, self.x, self.y, self.gens = wl["automaton"], wl["x"], wl["y"] * world, wl["gens"]
        self.P = O.PLANES[self.a]
        self.threads = host_threads(self.y)
        t0 = time.perf_counter()
        self.planes = O.init_bit_planes(self.x, self.y, self.P, wl["seed"], O.thresholds(wl["probs"]),
                                        threads=self.threads)
        self.init_s = time.perf_counter() - t0
        self.kind = "reference" if O.ref_available() else "port"
        if self.kind == "port":
            self.threads = 1

    def time(self, gens: int, threads: int) -> float:
        if self.kind == "reference":
            return self.O.ref_bench_planes64(self.a, self.planes, self.x, self.y, gens, threads)
        t0 = time.perf_counter()
        self.O.run_bit_planes(self.a, self.planes.reshape(-1), self.x, self.y, gens)
        return time.perf_counter() - t0

    def sample(self, target_s: float, threads: int) -> dict:
        probe = max(self.time(1, threads), 1e-4)
        gens = max(1, min(self.gens, int(target_s / probe)))
        secs = self.time(gens, threads)
        return {"value": self.x * self.y * gens / secs / 1e9, "gens": gens, "secs": secs, "threads": threads}

    def describe(self, s: dict) -> str:
        where = (f"{s['threads']} host threads, each the reference traverser on a {self.x}x{self.y // s['threads']} "
                 f"band of the {self.x}x{self.y} grid (a torus of its own)" if s["threads"] > 1 else
                 f"1 host thread, the whole {self.x}x{self.y} grid")
        what = ("Cellato CPU simple traverser, bit_planes layout, 64-bit words" if self.kind == "reference" else
                "C restatement of the bit-plane evaluator (oracle port)")
        full_s = s["secs"] * self.gens / s["gens"]
        return (f"{where}; {what}; {s['gens']} of the step's {self.gens} generations timed ({s['secs']:.2f} s), "
                f"a full step extrapolated at that rate to {full_s:.1f} s; host CPU {cpu_model()}")

    def standard_sample(self, target_s: float, rows: int = 64) -> dict:
        """One thread, the reference traverser with the standard layout (a byte
        per cell, the per-cell evaluator: Cellato's reference configuration) on
        the first `rows` rows of the grid as a torus of its own."""
        import numpy as np

        rows = min(rows, self.y)
        band = np.ascontiguousarray(self.planes[:, :rows, :])
        cells = self.O.unpack("bit_planes", band, self.x, rows, self.P, 32)
        probe = max(self.O.ref_bench(self.a, cells, 1, 1, layout="standard"), 1e-4)
        gens = max(1, min(self.gens, int(target_s / probe)))
        secs = self.O.ref_bench(self.a, cells, gens, 1, layout="standard")
        full_s = secs * self.gens / gens * self.y / rows
        return {"value": self.x * rows * gens / secs / 1e9, "unit": METRIC, "cores": 1,
                "sample": (f"1 host thread, Cellato CPU simple traverser, standard layout (one byte per cell), on a "
                           f"{self.x}x{rows} band of the {self.x}x{self.y} grid (a torus of its own); {gens} "
                           f"generations timed ({secs:.2f} s), a full step of the whole grid extrapolated at that "
                           f"rate to {full_s:.0f} s; host CPU {cpu_model()}")}

    def baseline(self, target_s: float) -> dict:
        """cpu_baseline of the B200 arm: the all-threads aggregate, one thread,
        and one thread with the reference's standard layout."""
        agg = self.sample(target_s, self.threads)
        one = self.sample(min(target_s, 4.0), 1) if self.threads > 1 else agg
        out = {"value": agg["value"], "unit": METRIC, "cores": agg["threads"], "kind": self.kind,
               "sample": self.describe(agg),
               "single_core": {"value": one["value"], "unit": METRIC, "cores": 1, "sample": self.describe(one)},
               "cpu_model": cpu_model()}
        if self.kind == "reference":
            out["single_core_standard_layout"] = self.standard_sample(min(target_s, 2.0))
        return out


def reference_arm(args, wl) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    ref = ReferenceSample(wl, world)
    for _ in range(args.warmup):
        ref.sample(0.5, ref.threads)
    samples = [ref.sample(2.0, ref.threads) for _ in range(args.steps)]
    gens = sum(s["gens"] for s in samples)
    secs = sum(s["secs"] for s in samples)
    value = ref.x * ref.y * gens / secs / 1e9
    one = ref.sample(2.0, 1) if ref.threads > 1 else samples[-1]
    base = {"value": value, "unit": METRIC, "cores": ref.threads, "kind": ref.kind,
            "sample": ref.describe(dict(samples[-1], gens=gens, secs=secs)),
            "single_core": {"value": one["value"], "unit": METRIC, "cores": 1, "sample": ref.describe(one)},
            "cpu_model": cpu_model()}
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": secs / gens * ref.gens * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u64", "data": "synthetic",
           "config": headline_config(wl, world),
           "sample": (f"each step times {samples[-1]['gens']} generations of the step's {ref.gens} on the "
                      f"benchmark grid; ms_per_step extrapolates the measured rate to the whole step"),
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


def bench_batch(cb, torch, stream, n: int, runs: int, automata=(0, 1, 2), temporal_steps: int = 0,
                tile_rows: int = 0) -> dict:
    specs = batch_workload(n, automata=automata)
    grids = []
    for i, (a, x, y, _) in enumerate(specs):
        g = cb.DeviceGrid(a, x, y)
        g.fill_random(1000 + i, batch_probs(cb, a), stream=stream)
        g.set_seed(5000 + i)
        grids.append(g)
    steps = [s for (_, _, _, s) in specs]
    batch = cb.Batch(grids, steps, temporal_steps=temporal_steps, tile_rows=tile_rows)
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
            "chunk_generations": temporal_steps or "library default", "tile_rows": tile_rows or "library default",
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
        # the median of five runs of the batched server (one Poisson stream each, the same
        # arrival times; the makespan is a few tenths of a second and which requests share a
        # round depends on host timing, so single runs vary, occasionally by 2x)
        runs = sorted((serve_stream(cb, specs, rate, False) for _ in range(5)), key=lambda r: r["throughput"])
        batched = dict(runs[2], throughput_of_runs=[r["throughput"] for r in runs])
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


class Ranks:
    """Barrier and max-over-ranks for the timed regions (no-ops on one rank)."""

    def __init__(self, torch, dist, world: int):
        self.torch, self.dist, self.world = torch, dist, world

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device="cuda")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())


def roofline(cb, a, name, x, y, P, plan, avg_launch_s, gens_per_launch, lop3_peak, traffic_key=True) -> dict:
    """The strip kernel against the measured integer-logic peak and the measured HBM copy peak."""
    cells = x * y
    bytes_per_launch = 2 * P * cells / 8  # read + write every plane once
    hbm_gbs = bytes_per_launch / avg_launch_s / 1e9
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs", FALLBACK_HBM_GBS)
    alu_per_word, shfl_per_word = cb.network_ops(a)
    if plan.get("rows_per_step", 1) == 1:  # one row per step: no pair evaluation
        alu_per_word += ROW_BY_ROW_EXTRA_OPS.get(a, 0)
    int_gops = alu_per_word * (cells / 32) * gens_per_launch / avg_launch_s / 1e9
    int_frac = int_gops / (lop3_peak / 1e9)
    hbm_frac = hbm_gbs / hbm_peak
    key = (f"pipe_kernel<{name},K={plan['temporal_steps']},V={plan['words_per_lane']},L={plan['levels_per_warp']},"
           f"R={plan['rows_per_step']}>@{x}x{y}")
    is_int = int_frac >= hbm_frac
    return {
        "bound": "int" if is_int else "hbm",
        "kernel": key,
        "achieved": int_gops if is_int else hbm_gbs,
        "peak": lop3_peak / 1e9 if is_int else hbm_peak,
        "unit": "Gop/s" if is_int else "GB/s",
        "frac": max(int_frac, hbm_frac),
        "traffic": traffic_for(key) if traffic_key else None,
        "peak_source": ("measured LOP3 issue rate (cb2_measure_lop3_peak, this run)" if is_int else
                        ("measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6.65 TB/s")),
        "int": {"achieved_gops": int_gops, "peak_gops": lop3_peak / 1e9, "frac": int_frac,
                "ops_per_word_per_generation": alu_per_word, "shuffles_per_word_per_generation": shfl_per_word},
        "hbm": {"achieved_gbs": hbm_gbs, "peak_gbs": hbm_peak, "frac": hbm_frac,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "avg_launch_ms": avg_launch_s * 1e3,
        "generations_per_launch": gens_per_launch,
    }


def best_plan_for_depth(cb, torch, grid, a, x, y, k: int, stream) -> dict:
    """Autotuning at a fixed temporal depth: every instantiated strip kernel of
    depth k, timed over 64 generations on the grid itself; the fastest plan."""
    best, best_ms = None, None
    for (kk, v, lv, r) in cb.variants(a):
        if kk != k:
            continue
        plan = dict(temporal_steps=k, words_per_lane=v, levels_per_warp=lv, rows_per_step=r)
        grid.run(k, **plan, stream=stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        grid.run(64, **plan, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        if best_ms is None or ms < best_ms:
            best, best_ms = plan, ms
    return best


def e2e_pipelined(cb, torch, grid, a, x, y, gens, run_kw, steps: int, stream) -> dict:
    """The e2e leg on one GPU, as a caller streaming a sequence of grids runs
    it: step i uploads the input image from pinned host memory into one of two
    device grids, runs `gens` generations and downloads the result into pinned
    host memory; the uploads and downloads go through cb2_grid_upload_async /
    cb2_grid_download_async on two copy streams, ordered by events, so step
    i+1's upload and step i-1's download overlap step i's run.  Timed from the
    first upload to the last download, on the device."""
    nbytes = cb.layout_bytes(a, "bit_planes", 64, x, y)
    host_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    host_out = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    grid.download("bit_planes", 64, stream=stream, out=host_in.numpy())
    host_img = cb.HostGrid(a, "bit_planes", 64, x, y, host_in.numpy())
    grids = [grid, cb.DeviceGrid(a, x, y)]
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()

    def pipeline(n):
        ev = lambda: torch.cuda.Event()  # noqa: E731
        downs = [None, None]
        for i in range(n):
            g = grids[i % 2]
            if downs[i % 2] is not None:  # the grid's previous result has left the device
                h2d.wait_event(downs[i % 2])
            g.upload_async(host_img, stream=h2d)
            up = ev()
            up.record(h2d)
            stream.wait_event(up)
            g.run(gens, **run_kw, stream=stream)
            ran = ev()
            ran.record(stream)
            d2h.wait_event(ran)
            g.download_async(host_out[i % 2].numpy(), stream=d2h)
            downs[i % 2] = ev()
            downs[i % 2].record(d2h)

    pipeline(2)  # warm-up (plans, second grid)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    f0.record(h2d)
    pipeline(steps)
    f1.record(d2h)
    f1.synchronize()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    ms = f0.elapsed_time(f1)
    grids[1].close()
    return {"value": x * y * gens * steps / (ms * 1e-3) / 1e9, "unit": METRIC, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "wall_s": wall,
            "path": "per step: cb2_grid_upload_async of the bit-plane image from pinned host memory, cb2_grid_run, "
                    "cb2_grid_download_async into pinned host memory; two device grids and two copy streams, so "
                    "step i+1's upload and step i-1's download overlap step i's run"}


def bench_layouts(cb, torch, wl, stream, steps: int = 3) -> dict:
    """The headline step through each host layout a Cellato grid can have
    (cb2_grid_upload / cb2_grid_download, synchronous, from and to pinned host
    memory): the device always runs the linear bit planes, and the bit_array
    and tiled_bit_planes images are converted on the device at upload and
    download.  Per layout: ms per step (upload, 1000 generations, download)
    and the boundary's share of it.  The standard layout (one byte per cell,
    4 GiB at 65536^2) is left out."""
    import numpy as np

    a, x, y, gens = wl["automaton"], wl["x"], wl["y"], wl["gens"]
    out = {"workload": wl["desc"], "steps": steps, "layouts": {}}
    with cb.DeviceGrid(a, x, y) as g:
        g.fill_random(wl["seed"], wl["probs"], stream=stream)
        for layout in ("bit_planes", "bit_array", "tiled_bit_planes"):
            n = cb.layout_bytes(a, layout, 64, x, y)
            h_in = torch.empty(n, dtype=torch.uint8, pin_memory=True)
            h_out = torch.empty(n, dtype=torch.uint8, pin_memory=True)
            g.download(layout, 64, stream=stream, out=h_in.numpy())
            img = cb.HostGrid(a, layout, 64, x, y, h_in.numpy())

            def copies():
                g.upload(img, stream=stream)
                g.download(layout, 64, stream=stream, out=h_out.numpy())
            copies()
            torch.cuda.synchronize()
            same = bool(np.array_equal(h_in.numpy(), h_out.numpy()))  # upload + download is the identity
            t0 = time.perf_counter()
            for _ in range(steps):
                copies()
            io_ms = (time.perf_counter() - t0) * 1e3 / steps
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            for _ in range(steps):
                g.upload(img, stream=stream)
                g.run(gens, stream=stream)
                g.download(layout, 64, stream=stream, out=h_out.numpy())
            e1.record(stream)
            e1.synchronize()
            step_ms = e0.elapsed_time(e1) / steps
            out["layouts"][layout] = {"ms_per_step": step_ms, "upload_download_ms": io_ms,
                                      "boundary_share": io_ms / step_ms, "host_bytes": n,
                                      "value": x * y * gens / (step_ms * 1e-3) / 1e9, "unit": METRIC,
                                      "round_trip_equal": same}
    return out


def measure(cb, torch, ranks, wl, args, rank, world, local_rank, stream, lop3_peak, depth: int = 0,
            e2e: bool = True) -> dict:
    """Times `args.steps` steps of workload `wl` (after `args.warmup` warm-up
    steps) with inputs resident in HBM, and, with `e2e`, the same steps through
    the public API with the bit planes copied from and to pinned host memory.
    depth > 0 fixes the temporal depth (the fastest kernel of that depth)."""
    a, x, y, gens = wl["automaton"], wl["x"], wl["y"], wl["gens"]
    name, P, _ = cb.automaton_info(a)
    cells = x * y
    tuned = None
    if world == 1:
        grid = cb.DeviceGrid(a, x, y)
        grid.fill_random(wl["seed"], wl["probs"], stream=stream)
        if depth:
            run_kw = best_plan_for_depth(cb, torch, grid, a, x, y, depth, stream)
            grid.fill_random(wl["seed"], wl["probs"], stream=stream)
        else:
            tuned = None if args.no_autotune else cb.autotune(a, x, y, budget_ms=4000)
            run_kw = {}
        plan = cb.plan(a, x, y, **run_kw)
    else:
        # one grid of world*y rows split into bands, one per rank (NCCL halo exchange per pass)
        from cellato_b200.bands import BandGrid

        if not args.no_autotune:
            tuned = cb.autotune(a, x, y, budget_ms=4000)
        grid = BandGrid(a, x, y * world, rank, world)
        grid.fill_random(wl["seed"], wl["probs"], stream=stream)
        # every rank must take the same passes (one halo exchange each): use rank 0's depth
        kt = torch.tensor([depth or grid.plan_k()], dtype=torch.int64, device="cuda")
        ranks.dist.broadcast(kt, 0)
        run_kw = {"temporal_steps": int(kt.item())}
        plan = cb.plan(a, x, y, **run_kw)
    k = plan["temporal_steps"]

    # ---- device-resident timing ----
    for _ in range(args.warmup):
        grid.run(gens, **run_kw, stream=stream)
    torch.cuda.synchronize()
    ranks.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_index(local_rank)) if local_rank == 0 else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        grid.run(gens, **run_kw, stream=stream)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ranks.barrier()
    clocks = sampler.stop() if sampler else None
    ms = ranks.max(e0.elapsed_time(e1))
    value = world * cells * gens * args.steps / (ms * 1e-3) / 1e9
    launches = launches_per_run(gens, k) * args.steps * (1 if world == 1 else 3)
    strip_launches = launches_per_run(gens, k) * args.steps
    roof = roofline(cb, a, name, x, y, P, plan, ms * 1e-3 / strip_launches, gens * args.steps / strip_launches,
                    lop3_peak)
    out = {"value": value, "unit": METRIC, "ms_per_step": ms / args.steps, "plan": plan, "autotuned": tuned,
           "roofline": roof, "clocks": clocks, "gpu_launches": launches}

    if e2e and world == 1:
        out["e2e"] = e2e_pipelined(cb, torch, grid, a, x, y, gens, run_kw, args.steps, stream)
    elif e2e:
        nbytes = cb.layout_bytes(a, "bit_planes", 64, x, y)
        host_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        host_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
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
        ranks.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        f1.synchronize()
        wall = time.perf_counter() - w0
        ranks.barrier()
        e2e_ms = ranks.max(f0.elapsed_time(f1))
        out["e2e"] = {"value": world * cells * gens * args.steps / (e2e_ms * 1e-3) / 1e9, "unit": METRIC,
                      "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "wall_s": ranks.max(wall),
                      "path": "band planes from pinned host memory + BandGrid.run (halo exchange overlapped with "
                              "the band interior, cb2_band_pass_at per pass) + band planes back, per rank"}
    if world == 1:
        grid.close()
    else:
        del grid
    torch.cuda.synchronize()
    return out


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
    ap.add_argument("--no-extra-workloads", action="store_true",
                    help="skip the WireWorld / Greenberg-Hastings lines and the per-depth lines")
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

    ranks = Ranks(torch, dist, world)
    stream = torch.cuda.current_stream()
    lop3_peak = cb.measure_lop3_peak()
    head = measure(cb, torch, ranks, wl, args, rank, world, local_rank, stream, lop3_peak)

    # the other single-grid workloads (WireWorld and Greenberg-Hastings 32768^2), and the headline
    # at each fixed temporal depth
    workloads, depths = None, None
    if world == 1 and not args.no_extra_workloads and args.workload == "gol-65536":
        workloads = {}
        for key in ("wire-32768", "excitable-32768"):
            workloads[key] = dict(measure(cb, torch, ranks, WORKLOADS[key], args, rank, world, local_rank, stream,
                                          lop3_peak), workload=WORKLOADS[key]["desc"])
        depth_args = argparse.Namespace(**dict(vars(args), steps=max(2, min(args.steps, 5)), warmup=3))
        depths = {"workload": wl["desc"], "steps": depth_args.steps, "warmup": depth_args.warmup,
                  "note": "each depth runs its fastest strip kernel, timed on the grid itself (autotuned per k)",
                  "autotuned": {"temporal_steps": head["plan"]["temporal_steps"], "value": head["value"],
                                "roofline_frac": head["roofline"]["frac"], "bound": head["roofline"]["bound"]}}
        for k in (1, 2, 4, 8):
            r = measure(cb, torch, ranks, wl, depth_args, rank, world, local_rank, stream, lop3_peak, depth=k,
                        e2e=False)
            depths[f"k={k}"] = {"value": r["value"], "unit": METRIC, "ms_per_step": r["ms_per_step"],
                                "plan": r["plan"], "roofline": r["roofline"], "clocks": r["clocks"]}

    layouts = None
    if world == 1 and not args.no_extra_workloads and args.workload == "gol-65536":
        layouts = bench_layouts(cb, torch, wl, stream)

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
        cpu = ReferenceSample(wl, world).baseline(args.cpu_seconds)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {
        "metric": METRIC, "value": head["value"], "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": headline_config(wl, world),
        "plan": head["plan"], "autotuned": head["autotuned"],
        "roofline": head["roofline"],
        "e2e": head["e2e"],
        "gpu_launches": head["gpu_launches"],
        "clocks": head["clocks"],
        "cpu_baseline": cpu,
        "workloads": workloads,
        "temporal_depths": depths,
        "layouts": layouts,
        "batched": batched,
        "batched_dsl": batched_dsl,
        "served": served,
        "served_dsl": served_dsl,
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
