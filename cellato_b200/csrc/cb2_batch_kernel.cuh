// cb2_batch_kernel.cuh -- the persistent batch kernel, templated on the rule
// set it dispatches to (internal).  cb2_batch.cu instantiates it over the
// hand-written networks; cb2_generic_batch.cu over those and the lowered
// DSL automata, whose window rules also read each chunk's generation and the
// grid's random seed.  The schedule it runs is described in cb2_batch.cu.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "cb2_batch.h"
#include "cb2_internal.h"
#include "cb2_pipe.cuh"

namespace cb2 {

constexpr int kBatchKMax = 8;  // longest chunk of a task of the kernel over every automaton

// Input rows a task keeps in flight: at least two groups of `rows`.
__host__ __device__ constexpr int batch_ring_depth(int rows) { return 2 * rows > kRingDepth ? 2 * rows : kRingDepth; }

// Shared memory of a task pipeline of P planes with `rows` rows per barrier
// over `warps` warps: the input ring plus two hand-off slots per warp boundary.
__host__ __device__ constexpr int batch_smem_words(int planes, int rows, int warps) {
    return (batch_ring_depth(rows) + 2 * rows * (warps - 1)) * planes * 32;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait until *p != 0; gives up early when another CTA failed.
__device__ __forceinline__ bool wait_flag(const unsigned* p, long long limit, const unsigned* error) {
    for (long long i = 0;; ++i) {
        if (ld_acquire(p) != 0) return true;
        if (i >= limit || ld_acquire(error) != 0) return false;
        __nanosleep(i < 32 ? 64 : 512);
    }
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// First generation of chunk c of a grid: nfull chunks of kmain, then the
// remainder in chunks of its binary digits, largest first (the host's split).
__device__ __forceinline__ int64_t chunk_start(const batch_grid_desc& g, int c) {
    if (c <= g.nfull) return g.t0 + (int64_t)c * g.kmain;
    int64_t t = g.t0 + (int64_t)g.nfull * g.kmain;
    int left = g.rem;
    for (int i = g.nfull; i < c; ++i) {
        const int k = 1 << (31 - __clz(left));
        t += k;
        left -= k;
    }
    return t;
}

// One chunk of K generations of one task on the whole CTA of WARPS warps: the
// level pipeline of pipe_run_rows with the K levels split over the warps,
// which divides a task's latency -- and with it the length of a grid's chain
// of chunks -- by the number of warps.  Chunks shorter than the CTA leave
// warps idle at the barriers.
template <class R, int K, int ROWS, int SMEM, int WARPS>
__device__ __forceinline__ void batch_run_task(const strip_task& t, const lane_geom<1>& geom, uint32_t* smem) {
    constexpr int L = K >= WARPS ? K / WARPS : 1;
    constexpr int W = K / L;
    constexpr int DEPTH = batch_ring_depth(ROWS);
    static_assert(pipe_rows_smem_words<R, K, 1, L, DEPTH, ROWS>() <= SMEM,
                  "task pipeline larger than the CTA's shared memory");
    if ((int)(threadIdx.x >> 5) < W)
        pipe_run_rows<R, K, 1, L, DEPTH, ROWS>(t, geom, smem);
    else
        pipe_rows_idle<K, L, ROWS>(t);
}

// One task of rule R with the chunk length k of the task (1, 2, 4, 8, 16 or 32, up to KMAX).
template <class R, int KMAX, int ROWS, int SMEM, int WARPS>
__device__ __forceinline__ void batch_run_rule(const strip_task& t, int k, const lane_geom<1>& geom, uint32_t* smem) {
    switch (k) {
    case 1: batch_run_task<R, 1, ROWS, SMEM, WARPS>(t, geom, smem); break;
    case 2: batch_run_task<R, 2, ROWS, SMEM, WARPS>(t, geom, smem); break;
    case 4: batch_run_task<R, 4, ROWS, SMEM, WARPS>(t, geom, smem); break;
    case 8:
        if constexpr (KMAX >= 8) batch_run_task<R, 8, ROWS, SMEM, WARPS>(t, geom, smem);
        break;
    case 16:
        if constexpr (KMAX >= 16) batch_run_task<R, 16, ROWS, SMEM, WARPS>(t, geom, smem);
        break;
    default:
        if constexpr (KMAX >= 32) batch_run_task<R, 32, ROWS, SMEM, WARPS>(t, geom, smem);
        break;
    }
}

// The persistent kernel.  D is the rule set: D::kWarps warps and D::kSmemWords
// shared words per CTA, and D::run(automaton, k, task, geom, smem) running one
// task.
template <class D>
__global__ void __launch_bounds__(D::kWarps * 32) batch_kernel(batch_args a) {
    __shared__ __align__(16) uint32_t smem[D::kSmemWords];
    __shared__ unsigned s_task;
    __shared__ int s_ok;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const unsigned ntasks = *a.ntasks;
    for (;;) {
        if (threadIdx.x == 0) s_task = ld_acquire(a.error) ? UINT_MAX : atomicAdd(a.head, 1u);
        __syncthreads();
        const unsigned t = s_task;
        if (t >= ntasks) break;  // the same for the whole CTA
        const batch_task task = a.tasks[t];
        const batch_grid_desc gd = a.grids[task.grid];
        // warp 0, lanes 0..8: the previous chunk's tasks on the 3x3 neighbouring tiles
        const unsigned* dep = a.task_done;
        if (task.dep_base >= 0) {
            const int j = lane < 9 ? lane : 4;  // lanes past the 3x3 tiles use the centre one
            const int dx = j % 3 - 1, dy = j / 3 - 1;
            dep += task.dep_base + wrap(task.ty + dy, task.nsy) * task.nsx + wrap(task.tx + dx, task.nsx);
        }
        if (warp == 0) {
            int ok = 1;
            if (task.dep_base >= 0 && lane < 9) ok = wait_flag(dep, a.spin_limit, a.error);
            ok = __all_sync(kFullMask, ok);
            if (lane == 0) {
                s_ok = ok;
                if (!ok) atomicCAS(a.error, 0u, t + 1);
            }
        }
        __syncthreads();
        if (!s_ok) break;
        if (task.dep_base >= 0) (void)ld_acquire(dep);  // acquire in every thread
        strip_task st;
        st.in = gd.buf[task.chunk & 1];
        st.out = gd.buf[(task.chunk & 1) ^ 1];
        st.plane_words = gd.plane_words;
        st.t0 = D::kTimed ? chunk_start(gd, task.chunk) : 0;
        st.seed = gd.seed;
        st.y_global0 = 0;
        st.global_h = gd.h;
        st.wd = gd.wd;
        st.h = gd.h;
        lane_geom<1> geom;
        st.y0 = task.y0;
        st.ny = task.rows;
        if (task.groups > 0) {
            st.x0 = 0;
            st.nx = gd.wd;
            geom = group_geom(st, task.groups, lane);
        } else {
            // lowered rules: tiles start at an odd column, so that stochastic
            // rules' lanes pair up on groups of 64 cells (the last tile owns
            // column 0 through the wrap)
            const int shift = D::kTimed && gd.automaton >= kNumBuiltin ? 1 : 0;
            st.x0 = task.tx * 30 + shift;
            st.nx = min(30, gd.wd - task.tx * 30);
            geom = task.groups < 0 ? band_geom(st, -task.groups, lane) : strip_geom<1>(st, lane);
        }
        D::run(gd.automaton, task.k, st, geom, smem);
        __threadfence();  // this thread's stores are visible GPU-wide before the flag
        __syncthreads();  // every warp's stores are done; smem and s_task are free again
        if (threadIdx.x == 0) atomicExch(a.task_done + t, 1u);
    }
}

} // namespace cb2
