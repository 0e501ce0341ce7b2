"""TEST AND MEASUREMENT INFRASTRUCTURE ONLY: the reference's own CUDA kernels on this GPU.

Times Cellato's CUDA ``simple`` and ``temporal`` bit-plane traversers
(oracle/_ref/libcellato_ref_cuda.so, built by oracle/Makefile from the
reference headers, see ref_cuda_shim.cu) on the headline workloads, next to
this project's strip kernels on the same input, and checks that both produce
the same cells.  The reference's temporal kernel needs the grid's width in
64-bit words to be a multiple of 30 (32-word blocks minus one halo word each
side, traversers/cuda/temporal.hpp:44-59) and its height a multiple of the
effective tile height, so it runs on the nearest smaller grid of that shape;
the simple kernel and this project run on the exact bench size too.

    python -m oracle.ref_cuda_bench [--quick] [--dsl] [--only NAME[,NAME...]]

prints one JSON object per line (sweep points, then a summary per workload).
With --dsl the workloads are the lowered DSL automata (every bundled
automaton without a hand-written network, and the two stochastic examples)
at 16384 x 16384, uniform states, and this project's plan is both the
default and the autotuned one.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libcellato_ref_cuda.so")

WORKLOADS = [  # the bench's three single-grid workloads (automaton, x, y, probabilities, seed)
    ("game-of-life", 0, 65536, 65536, [0.65, 0.35], 42),
    ("wire", 1, 32768, 32768, [0.60, 0.05, 0.05, 0.30], 42),
    ("excitable", 2, 32768, 32768, [0.125] * 8, 42),
]
DSL = ["brian", "critters", "cyclic", "forest-fire", "fluid", "maze", "traffic", "lightning-forest", "noisy-life"]
# compiled temporal option set of ref_cuda_shim.cu
KS, TILES, BLOCKS = (2, 4, 8, 12, 16), (16, 32, 64), (4, 8, 16)
SMEM_LIMIT = 48 * 1024  # the temporal kernel asks for no more than the default dynamic shared memory


def load():
    lib = ctypes.CDLL(LIB)
    lib.ref_cuda_run.restype = ctypes.c_int
    lib.ref_cuda_run.argtypes = [ctypes.c_int] * 9 + [ctypes.c_void_p, ctypes.c_void_p,
                                                      ctypes.POINTER(ctypes.c_float), ctypes.c_char_p, ctypes.c_int]
    return lib


def ref_run(lib, a, trav, x, y, warm, steps, k, tile, block_y, planes: np.ndarray):
    out = np.empty_like(planes)
    ms = ctypes.c_float()
    err = ctypes.create_string_buffer(512)
    rc = lib.ref_cuda_run(a, trav, x, y, warm, steps, k, tile, block_y, planes.ctypes.data, out.ctypes.data,
                          ctypes.byref(ms), err, 512)
    if rc:
        raise RuntimeError(err.value.decode(errors="replace") or f"ref_cuda_run returned {rc}")
    return out, ms.value


def temporal_configs(P: int):
    for k in KS:
        for tile in TILES:
            for by in BLOCKS:
                if tile - 2 * k <= 0 or tile % by or 2 * tile * 32 * P * 8 > SMEM_LIMIT:
                    continue
                yield k, tile, by


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="small grids, for a smoke check of the harness")
    ap.add_argument("--dsl", action="store_true", help="the lowered DSL automata instead of the headline three")
    ap.add_argument("--only", default="", help="comma-separated workloads (automaton names) to run")
    args = ap.parse_args()
    import torch

    import cellato_b200 as cb
    from oracle import oracle as O

    lib = load()
    workloads = WORKLOADS
    if args.dsl:
        workloads = []
        for n in DSL:
            states = cb.automaton_info(n)[2]
            probs = [0.5, 0.25, 0.25] if states == 3 else [1.0 / states] * states  # exact binary fractions
            workloads.append((n, O.ref_automaton(n), 16384, 16384, probs, 42))
    if args.only:
        keep = set(args.only.split(","))
        workloads = [w for w in workloads if w[0] in keep]
    for name, a, X, Y, probs, seed in workloads:
        if args.quick:
            X, Y = 30720, 1024  # a multiple of 32 and of 30 words
        _, P, _ = cb.automaton_info(name)

        def planes_for(x, y):
            with cb.DeviceGrid(name, x, y) as g:
                g.fill_random(seed, probs)
                return np.ascontiguousarray(g.download("bit_planes", 64).data)

        def ours(x, y, planes, steps):
            with cb.DeviceGrid(name, x, y) as g:
                g.upload(cb.HostGrid(name, "bit_planes", 64, x, y, planes))
                g.run(32)  # warm-up on a copy: the timed run starts from the same planes below
                g.upload(cb.HostGrid(name, "bit_planes", 64, x, y, planes))
                g.time_step = 0
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                g.run(steps)
                e1.record()
                e1.synchronize()
                return np.ascontiguousarray(g.download("bit_planes", 64).data), e0.elapsed_time(e1)

        summary = {"workload": name, "x": X, "y": Y}
        # -- reference simple kernel, exact size ------------------------------------------
        planes = planes_for(X, Y)
        steps_simple = 8 if args.quick else 64
        _, ms = ref_run(lib, a, 0, X, Y, 2, steps_simple, 0, 0, 8, planes)  # timed after 2 warm-up launches
        # Cells from a run without warm-up: the reference's run() numbers generations from 0 on every
        # call (traversers/cuda/simple.cuh:60-77), which time-dependent rules read.
        ref_out, _ = ref_run(lib, a, 0, X, Y, 0, steps_simple, 0, 0, 8, planes)
        mine, my_ms = ours(X, Y, planes, steps_simple)
        simple = {"kernel": "reference cuda::simple (bit_planes, u64, block 32x8)", "x": X, "y": Y,
                  "steps": steps_simple, "gcells_s": X * Y * steps_simple / (ms * 1e-3) / 1e9,
                  "same_cells_as_ours": bool(np.array_equal(ref_out, mine))}
        print(json.dumps({"workload": name, "simple": simple}), flush=True)
        summary["reference_simple"] = simple
        # -- reference temporal kernel: sweep the compiled options -------------------------
        xt = (X // (30 * 64)) * 30 * 64
        best = None
        sweep_steps = 48  # a multiple of every compiled k
        for k, tile, by in temporal_configs(P):
            eff = tile - 2 * k
            yt = (Y // eff) * eff
            tp = planes_for(xt, yt)
            try:
                _, ms = ref_run(lib, a, 1, xt, yt, 2 * k, sweep_steps, k, tile, by, tp)
            except RuntimeError as e:
                print(json.dumps({"workload": name, "temporal": [k, tile, by], "error": str(e)}), flush=True)
                continue
            rate = xt * yt * sweep_steps / (ms * 1e-3) / 1e9
            print(json.dumps({"workload": name, "temporal": [k, tile, by], "x": xt, "y": yt, "gcells_s": rate}),
                  flush=True)
            if best is None or rate > best[0]:
                best = (rate, k, tile, by, yt)
        rate, k, tile, by, yt = best
        steps_t = 48 if args.quick else 480
        tp = planes_for(xt, yt)
        # Warm-ups of an even number of launches: the reference's run() always starts from the
        # grid given to init() (traversers/cuda/temporal.cuh:151-152), which holds the current
        # state again only after an even number of launches.  Cells again from a run without one.
        _, ms = ref_run(lib, a, 1, xt, yt, 2 * k, steps_t, k, tile, by, tp)
        ref_out, _ = ref_run(lib, a, 1, xt, yt, 0, steps_t, k, tile, by, tp)
        mine, my_ms_t = ours(xt, yt, tp, steps_t)
        temporal = {"kernel": f"reference cuda::temporal (bit_planes, u64), best compiled option k={k}, "
                              f"tile_y={tile}, block 32x{by}", "x": xt, "y": yt, "steps": steps_t,
                    "gcells_s": xt * yt * steps_t / (ms * 1e-3) / 1e9,
                    "same_cells_as_ours": bool(np.array_equal(ref_out, mine))}
        summary["reference_temporal"] = temporal
        # -- this project's strip kernels, same sizes, default plan ---------------------
        n_ours = 480 if not args.quick else 48
        _, my_ms = ours(X, Y, planes, n_ours)
        summary["ours"] = {"kernel": "cellato_b200 strip kernels, default plan " + json.dumps(cb.plan(name, X, Y)),
                           "x": X, "y": Y, "steps": n_ours, "gcells_s": X * Y * n_ours / (my_ms * 1e-3) / 1e9}
        if args.dsl:
            tuned = cb.autotune(name, X, Y, budget_ms=3000)
            _, my_ms = ours(X, Y, planes, n_ours)
            summary["ours_autotuned"] = {"plan": tuned, "gcells_s": X * Y * n_ours / (my_ms * 1e-3) / 1e9}
        summary["speedup_vs_reference_temporal"] = summary["ours"]["gcells_s"] / temporal["gcells_s"]
        summary["speedup_vs_reference_simple"] = summary["ours"]["gcells_s"] / simple["gcells_s"]
        print(json.dumps({"summary": summary}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
