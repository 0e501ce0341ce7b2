// cb2_launch.cuh -- the strip kernel as launched, shared by the translation
// units that instantiate it: cb2_kernels.cu (the hand-written networks) and
// cb2_generic.cu (the lowered DSL automata).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cb2_internal.h"
#include "cb2_pipe.cuh"

namespace cb2 {

// One launch: K generations over output rows [y_base, y_base + rows_out),
// strip tasks of nsx columns x nsy row tiles, one CTA each.
struct strip_launch {
    const uint32_t* in;
    uint32_t* out;
    int64_t plane_words;
    int32_t wd, h;
    int32_t nsx, nsy, tile_rows;
    int32_t y_base, rows_out;  // output rows [y_base, y_base + rows_out)
    int64_t t0;                // generation of the input
    uint64_t seed;             // random seed of stochastic rules
    int64_t y_global0;         // global row of row 0 of the planes (a band's offset)
    int64_t global_h;          // rows of the whole grid
};

template <class R, int K, int V, int L, int RPS>
__global__ void __launch_bounds__(32 * (K / L)) pipe_kernel(strip_launch a) {
    extern __shared__ __align__(16) uint32_t smem[];
    constexpr int own = 32 * V - 2;
    const int task = blockIdx.x;
    const int sx = task % a.nsx, sy = task / a.nsx;
    strip_task t;
    t.in = a.in;
    t.out = a.out;
    t.plane_words = a.plane_words;
    t.wd = a.wd;
    t.h = a.h;
    // A rule that draws random numbers, one word per lane: strips start at an
    // odd column, so that lanes 2m and 2m+1 hold the two halves of a group of
    // 64 cells and split its draws (the last strip owns column 0 through the
    // wrap; on an odd width the lanes past the wrap draw alone).
    const int shift = draws_of<R>::value && V == 1 ? 1 : 0;
    t.x0 = sx * own + shift;
    t.nx = min(own, a.wd - sx * own);
    t.y0 = a.y_base + sy * a.tile_rows;
    t.ny = min(a.tile_rows, a.y_base + a.rows_out - t.y0);
    t.t0 = a.t0;
    t.seed = a.seed;
    t.y_global0 = a.y_global0;
    t.global_h = a.global_h;
    if constexpr (RPS > 1)
        pipe_run_rows<R, K, V, L, kRingDepth, RPS>(t, smem);  // RPS rows per barrier
    else if constexpr (L == K)
        warp_run<R, K, V, kRingDepth>(t, strip_geom<V>(t, threadIdx.x & 31), smem);  // one warp, skewed levels
    else
        pipe_run<R, K, V, L, kRingDepth>(t, smem);
}

template <class R, int K, int V, int L, int RPS = 1>
static strip_variant make_variant() {
    int words;
    if constexpr (RPS > 1)
        words = pipe_rows_smem_words<R, K, V, L, kRingDepth, RPS>();
    else if constexpr (L == K)
        words = warp_smem_words<R, V, kRingDepth>();
    else
        words = pipe_smem_words<R, K, V, L, kRingDepth>();
    return strip_variant{K, V, L, RPS, (const void*)pipe_kernel<R, K, V, L, RPS>, 32 * (K / L), 4 * words};
}

} // namespace cb2
