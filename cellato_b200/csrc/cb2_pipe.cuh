// cb2_pipe.cuh -- the strip wavefront split across the warps of a CTA.
//
// Keeping all K levels of the temporal wavefront in the registers of one warp
// makes the register count -- and with it the number of resident warps --
// grow with K.  pipe_run splits the K levels over the W = K / L warps of a
// CTA: warp w owns levels [w*L, (w+1)*L) of the same strip and the CTA
// advances in lock step, one row per step:
//
//   warp 0      takes the next input row from a shared-memory ring that
//               cp.async keeps DEPTH rows ahead (global loads never block a
//               register), pushes it through its L levels
//   warp w > 0  takes the row warp w-1 produced in the previous step from a
//               double-buffered shared-memory slot, pushes it through its L
//               levels
//   warp W-1    writes the finished row (generation t+K) to global memory
//
// One __syncthreads per step separates the slot a warp writes from the slot
// its successor reads.  pipe_run_rows is the same pipeline with RPS rows per
// step (RPS-row slots, one barrier per RPS rows).  The row bookkeeping is the single-warp wavefront's:
// input row r (sweep coordinates) leaves warp W-1 at step r + W - 1 as output
// row r - K, so rows before the 2K-row warm-up are computed but never stored.
#pragma once

#include <cstdint>
#include <type_traits>

#include "cb2_strip.cuh"

namespace cb2 {

template <int V>
struct pipe_vec;  // one lane's V words as a single shared-memory access
template <>
struct pipe_vec<1> {
    using type = uint32_t;
};
template <>
struct pipe_vec<2> {
    using type = uint2;
};
template <>
struct pipe_vec<4> {
    using type = uint4;
};

// Shared memory of one CTA in 32-bit words.
template <class R, int K, int V, int L, int DEPTH>
constexpr int pipe_smem_words() {
    return (DEPTH + 2 * (K / L - 1)) * R::P * 32 * V;
}

__device__ __forceinline__ void cp_async4(uint32_t* smem, const uint32_t* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A row slot in shared memory: plane p, lane l, word i at ((p*32)+l)*V + i.
template <class R, int V>
__device__ __forceinline__ void slot_read(const uint32_t* slot, int lane, uint32_t (&row)[V][R::P]) {
    using vec = typename pipe_vec<V>::type;
#pragma unroll
    for (int p = 0; p < R::P; ++p) {
        const vec v = reinterpret_cast<const vec*>(slot)[p * 32 + lane];
        const uint32_t* w = reinterpret_cast<const uint32_t*>(&v);
#pragma unroll
        for (int i = 0; i < V; ++i) row[i][p] = w[i];
    }
}

template <class R, int V>
__device__ __forceinline__ void slot_write(uint32_t* slot, int lane, const uint32_t (&row)[V][R::P]) {
    using vec = typename pipe_vec<V>::type;
#pragma unroll
    for (int p = 0; p < R::P; ++p) {
        vec v;
        uint32_t* w = reinterpret_cast<uint32_t*>(&v);
#pragma unroll
        for (int i = 0; i < V; ++i) w[i] = row[i][p];
        reinterpret_cast<vec*>(slot)[p * 32 + lane] = v;
    }
}

// A row read from the input ring enters the first level in the rule's
// working encoding (encode_states; the identity for most rules).
template <class R, int V>
__device__ __forceinline__ void input_row(const uint32_t* slot, int lane, uint32_t (&row)[V][R::P]) {
    slot_read<R, V>(slot, lane, row);
#pragma unroll
    for (int i = 0; i < V; ++i) encode_states<R>(row[i]);
}

// Runs one strip task on the whole CTA (W = K / L warps, all active).
// `smem` holds pipe_smem_words<R, K, V, L, DEPTH>() words, 16-byte aligned.
template <class R, int K, int V, int L, int DEPTH>
__device__ __forceinline__ void pipe_run(const strip_task& t, uint32_t* smem) {
    static_assert(!R::kWindow, "window rules run in pipe_run_rows");
    static_assert(K % L == 0, "levels per warp must divide K");
    static_assert(K <= 32, "the one-word halo of a strip covers at most 32 generations");
    static_assert(DEPTH >= 2, "input ring of at least two rows");
    constexpr int W = K / L;
    constexpr int P = R::P;
    constexpr int SLOT = P * 32 * V;  // words per row slot
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const lane_geom<V> geom = strip_geom<V>(t, lane);

    strip_state<R, L, V> s;
#pragma unroll
    for (int g = 0; g < L; ++g)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int i = 0; i < V; ++i) {
#pragma unroll
                for (int k = 0; k < R::NH; ++k) s.h[g][q][i][k] = 0;
#pragma unroll
                for (int p = 0; p < P; ++p) s.c[g][q][i][p] = 0;
            }

    uint32_t* ring = smem;                  // DEPTH input rows (warp 0)
    uint32_t* hand = smem + DEPTH * SLOT;   // 2 slots per warp boundary
    const int total = t.ny + 2 * K;         // rows entering warp 0
    const int steps = total + W - 1;

    // Warp 0 keeps DEPTH-1 input rows in flight.
    int lr = 0;
    auto issue = [&](int r) {
        if (r < total) {
            const uint32_t* base = t.in + (int64_t)lr * t.wd;
            uint32_t* dst = ring + (r % DEPTH) * SLOT;
#pragma unroll
            for (int p = 0; p < P; ++p)
#pragma unroll
                for (int i = 0; i < V; ++i)
                    cp_async4(dst + (p * 32 + lane) * V + i, base + p * t.plane_words + geom.col[i]);
            lr = lr + 1 == t.h ? 0 : lr + 1;
        }
        cp_async_commit();  // empty groups keep the count uniform
    };
    if (warp == 0) {
        lr = (t.y0 - K) % t.h;
        if (lr < 0) lr += t.h;
#pragma unroll
        for (int r = 0; r < DEPTH - 1; ++r) issue(r);
    } else {
        // the first reads of every hand-off slot see zeros (warm-up rows)
        for (int j = lane; j < 2 * SLOT; j += 32) hand[(warp - 1) * 2 * SLOT + j] = 0;
    }
    __syncthreads();

    auto step = [&](int st, auto parity) {
        constexpr int Q = decltype(parity)::value;
        uint32_t row[V][P];
        if (warp == 0) {
            issue(st + DEPTH - 1);
            cp_async_wait<DEPTH - 1>();
            if (st < total) input_row<R, V>(ring + (st % DEPTH) * SLOT, lane, row);
            else
#pragma unroll
                for (int i = 0; i < V; ++i)
#pragma unroll
                    for (int p = 0; p < P; ++p) row[i][p] = 0;
        } else {
            slot_read<R, V>(hand + ((warp - 1) * 2 + (st & 1)) * SLOT, lane, row);
        }
        strip_push<R, L, V, Q>(s, row, geom.src_l, geom.src_r);
        if (warp == W - 1) {
            const int r0 = st - (W - 1);  // input row whose result leaves now
            if (r0 >= 2 * K && r0 < total) strip_store<R, V>(t, geom, r0 - 2 * K, row);
        } else {
            slot_write<R, V>(hand + (warp * 2 + ((st + 1) & 1)) * SLOT, lane, row);
        }
        __syncthreads();
    };
    for (int st = 0; st < steps; st += 2) {
        step(st, std::integral_constant<int, 0>{});
        if (st + 1 < steps) step(st + 1, std::integral_constant<int, 1>{});
    }
    if (warp == 0) cp_async_wait<0>();
}

// Shared memory of pipe_run_rows in 32-bit words: the input ring plus two
// RPS-row hand-off slots per warp boundary.
template <class R, int K, int V, int L, int DEPTH, int RPS>
__host__ __device__ constexpr int pipe_rows_smem_words() {
    return (DEPTH + 2 * RPS * (K / L - 1)) * R::P * 32 * V;
}

// pipe_run with RPS (even) rows per step: every warp pushes RPS consecutive
// rows through its levels between two barriers, which divides the barriers
// and the per-step bookkeeping per row by RPS.  Row j of a step uses level
// slot j & 1, so no step parity is needed.  cp.async groups hold RPS rows;
// the ring of DEPTH rows keeps DEPTH / RPS - 1 groups in flight.
template <class R, int K, int V, int L, int DEPTH, int RPS>
__device__ __forceinline__ void pipe_run_rows(const strip_task& t, const lane_geom<V>& geom, uint32_t* smem) {
    static_assert(K % L == 0, "levels per warp must divide K");
    static_assert(K <= 32, "the one-word halo of a strip covers at most 32 generations");
    static_assert(RPS >= 2 && RPS % 2 == 0, "an even number of rows per step");
    static_assert(DEPTH % RPS == 0 && DEPTH / RPS >= 2, "a ring of at least two groups of rows");
    constexpr int W = K / L;
    constexpr int P = R::P;
    constexpr int SLOT = P * 32 * V;  // words per row
    constexpr int G = DEPTH / RPS;    // groups of RPS rows in the ring
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    strip_state<R, L, V> s;
#pragma unroll
    for (int g = 0; g < L; ++g)
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int i = 0; i < V; ++i) {
#pragma unroll
                for (int k = 0; k < R::NH; ++k) s.h[g][q][i][k] = 0;
#pragma unroll
                for (int p = 0; p < P; ++p) s.c[g][q][i][p] = 0;
            }
    // A stochastic rule keys its streams once per level (warp w's level g runs
    // generation t0 + w*L + g for every row of the task), and with one word per
    // lane, lanes 2m and 2m+1 split the draws of a group of 64 cells when every
    // pair of the warp holds the two halves of one group in one row
    // (cell_ctx::paired; with strips starting at odd columns, all warps but
    // those past the wrap of an odd width).
    bool paired = false;
    // The global row each pushed row's first level outputs, kept as running
    // local (these planes, wrap at t.h) and global (wrap at the grid's rows)
    // counters: no division per row.  The first row pushed (sweep
    // -warp*(RPS+L), possibly a warm-up row of a later warp) outputs local row
    // y0 + yoff - K - 1 + sweep; a local wrap resyncs the global row to the
    // planes' offset.  Levels map their rows in global rows (row_ctx): a band's
    // local wrap only happens in rows no output depends on, since its ghost
    // rows are at least K deep.
    int64_t ylocal = 0, yglob = 0, yshift = 0, gh = 1;
    if constexpr (R::kWindow) {
        gh = t.global_h;
        const int64_t s0 = (int64_t)t.y0 + geom.yoff - K - 1 - (int64_t)warp * (RPS + L);
        ylocal = ((s0 % t.h) + t.h) % t.h;
        yshift = ((t.y_global0 % gh) + gh) % gh;
        yglob = (ylocal + yshift) % gh;
#pragma unroll
        for (int g = 0; g < L; ++g) s.rows.gm[g] = g % gh;
    }
    // branch-free, like the row pushes around it (a branch splits their code)
    auto next_row = [&]() {
        const bool wrap = ylocal + 1 == t.h;
        ylocal = wrap ? 0 : ylocal + 1;
        const int64_t yn = yglob + 1 == gh ? 0 : yglob + 1;
        yglob = wrap ? yshift : yn;
    };
    if constexpr (draws_of<R>::value) {
#pragma unroll
        for (int g = 0; g < L; ++g)
#pragma unroll
            for (int i = 0; i < V; ++i) R::init_keys(s.keys[g][i], t.t0 + (int64_t)warp * L + g, geom.col[i], t.seed);
        if constexpr (V == 1) {
            const long long pc = __shfl_xor_sync(kFullMask, (long long)geom.col[0], 1);
            const int py = __shfl_xor_sync(kFullMask, geom.yoff, 1);
            paired = __all_sync(kFullMask, ((long long)geom.col[0] ^ 1) == pc && py == geom.yoff);
        }
    }

    uint32_t* ring = smem;
    uint32_t* hand = smem + DEPTH * SLOT;  // boundary b, parity q: hand + (2b + q) * RPS * SLOT
    const int total = t.ny + 2 * K;
    const int steps = (total + RPS - 1) / RPS + W - 1;

    int lr = 0;
    auto issue = [&](int g) {  // rows [g*RPS, (g+1)*RPS) as one group
#pragma unroll
        for (int j = 0; j < RPS; ++j) {
            const int r = g * RPS + j;
            if (r < total) {
                const uint32_t* base = t.in + (int64_t)lr * t.wd;
                uint32_t* dst = ring + (r % DEPTH) * SLOT;
#pragma unroll
                for (int p = 0; p < P; ++p)
#pragma unroll
                    for (int i = 0; i < V; ++i)
                        cp_async4(dst + (p * 32 + lane) * V + i, base + p * t.plane_words + geom.col[i]);
                lr = lr + 1 == t.h ? 0 : lr + 1;
            }
        }
        cp_async_commit();
    };
    if (warp == 0) {
        lr = (t.y0 + geom.yoff - K) % t.h;  // a lane of a narrow grid's row group starts at its own rows
        if (lr < 0) lr += t.h;
#pragma unroll
        for (int g = 0; g < G - 1; ++g) issue(g);
    } else {
        for (int j = lane; j < 2 * RPS * SLOT; j += 32) hand[(warp - 1) * 2 * RPS * SLOT + j] = 0;
    }
    __syncthreads();

    // The rows, with the generation of this warp's first level.  A rule that
    // branches on the generation's parity (alternate_algorithms) gets one copy
    // of the loop per parity of the task's first generation, chosen once per
    // CTA: with an even number of levels per warp every level's parity is then
    // a compile-time constant and the branch folds.
    auto sweep = [&](auto parity) {
        constexpr int PAR = decltype(parity)::value;
        [[maybe_unused]] const int64_t tbase = (PAR < 0 ? t.t0 : ((t.t0 & ~(int64_t)1) | PAR)) + (int64_t)warp * L;
        for (int st = 0; st < steps; ++st) {
            uint32_t rows[RPS][V][P];
            if (warp == 0) {
                issue(st + G - 1);
                cp_async_wait<G - 1>();
#pragma unroll
                for (int j = 0; j < RPS; ++j) {
                    const int r = RPS * st + j;
                    if (r < total) {
                        input_row<R, V>(ring + (r % DEPTH) * SLOT, lane, rows[j]);
                    } else {
#pragma unroll
                        for (int i = 0; i < V; ++i)
#pragma unroll
                            for (int p = 0; p < P; ++p) rows[j][i][p] = 0;
                    }
                }
            } else {
                const uint32_t* in = hand + ((warp - 1) * 2 + (st & 1)) * RPS * SLOT;
#pragma unroll
                for (int j = 0; j < RPS; ++j) slot_read<R, V>(in + j * SLOT, lane, rows[j]);
            }
#pragma unroll
            for (int j = 0; j < RPS; j += 2) {
                if constexpr (R::kWindow) {
                    // warp w's chain receives sweep row RPS*st + j - w*(RPS + L) (warp w-1's
                    // output of the previous step, L rows behind its input); a lane of a
                    // narrow grid's row group sweeps from its own first row
                    row_ctx rc{tbase, yglob, gh, t.seed, paired};
                    next_row();
                    strip_push<R, L, V, 0>(s, rows[j], geom.src_l, geom.src_r, &geom, &rc);
                    rc.y = yglob;
                    next_row();
                    strip_push<R, L, V, 1>(s, rows[j + 1], geom.src_l, geom.src_r, &geom, &rc);
                } else if constexpr (has_pairs<R>::value) {
                    strip_push2<R, L, V>(s, rows[j], rows[j + 1], geom.src_l, geom.src_r);
                } else {
                    strip_push<R, L, V, 0>(s, rows[j], geom.src_l, geom.src_r);
                    strip_push<R, L, V, 1>(s, rows[j + 1], geom.src_l, geom.src_r);
                }
            }
            if (warp == W - 1) {
                const int r0 = RPS * (st - (W - 1));  // input rows whose results leave now
#pragma unroll
                for (int j = 0; j < RPS; ++j)
                    if (r0 + j >= 2 * K && r0 + j < total) strip_store<R, V>(t, geom, r0 + j - 2 * K, rows[j]);
            } else {
                uint32_t* out = hand + (warp * 2 + ((st + 1) & 1)) * RPS * SLOT;
#pragma unroll
                for (int j = 0; j < RPS; ++j) slot_write<R, V>(out + j * SLOT, lane, rows[j]);
            }
            __syncthreads();
        }
    };
    if constexpr (parity_of<R>::value && L % 2 == 0) {
        if (t.t0 & 1)  // the same for every warp of the CTA: the barriers in sweep stay uniform
            sweep(std::integral_constant<int, 1>{});
        else
            sweep(std::integral_constant<int, 0>{});
    } else {
        sweep(std::integral_constant<int, -1>{});
    }
    if (warp == 0) cp_async_wait<0>();
}

// pipe_run_rows over the strip geometry of the task.
template <class R, int K, int V, int L, int DEPTH, int RPS>
__device__ __forceinline__ void pipe_run_rows(const strip_task& t, uint32_t* smem) {
    pipe_run_rows<R, K, V, L, DEPTH, RPS>(t, strip_geom<V>(t, threadIdx.x & 31), smem);
}

// The barriers of pipe_run_rows<R, K, V, L, DEPTH, RPS> for a warp of the
// CTA beyond its K / L pipeline warps (a CTA sized for longer chains running
// a short one): it takes part in every __syncthreads and touches nothing.
template <int K, int L, int RPS>
__device__ __forceinline__ void pipe_rows_idle(const strip_task& t) {
    const int steps = (t.ny + 2 * K + RPS - 1) / RPS + K / L - 1;
    __syncthreads();
    for (int st = 0; st < steps; ++st) __syncthreads();
}

// Shared memory of one warp-strip (skewed single-warp kernel) in 32-bit words.
template <class R, int V, int DEPTH>
constexpr int warp_smem_words() {
    return DEPTH * R::P * 32 * V;
}

// Runs one strip task on one warp with all K levels in registers, in the
// skewed order of skewed_step: every level of a step is independent, so a
// warp has K*V independent chains to issue from.  Input rows stream through
// a cp.async ring of DEPTH rows in `smem` (warp_smem_words words); there is
// no barrier.  A row entering at step s leaves level K-1 at step s+K-1 as
// the row K rows above it: output sweep row s - 2K + 1.
template <class R, int K, int V, int DEPTH>
__device__ __forceinline__ void warp_run(const strip_task& t, const lane_geom<V>& geom, uint32_t* smem) {
    static_assert(!R::kWindow, "window rules run in pipe_run_rows");
    constexpr int P = R::P;
    constexpr int SLOT = P * 32 * V;
    const int lane = threadIdx.x & 31;

    strip_state<R, K, V> s;
    uint32_t pend[K][V][P];
#pragma unroll
    for (int g = 0; g < K; ++g)
#pragma unroll
        for (int i = 0; i < V; ++i) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
#pragma unroll
                for (int k = 0; k < R::NH; ++k) s.h[g][q][i][k] = 0;
#pragma unroll
                for (int p = 0; p < P; ++p) s.c[g][q][i][p] = 0;
            }
#pragma unroll
            for (int p = 0; p < P; ++p) pend[g][i][p] = 0;
        }

    const int total = t.ny + 2 * K;  // input rows
    const int steps = total + K - 1;
    int lr = (t.y0 + geom.yoff - K) % t.h;  // this lane's next input row
    if (lr < 0) lr += t.h;
    auto issue = [&](int r) {
        if (r < total) {
            const uint32_t* base = t.in + (int64_t)lr * t.wd;
            uint32_t* dst = smem + (r % DEPTH) * SLOT;
#pragma unroll
            for (int p = 0; p < P; ++p)
#pragma unroll
                for (int i = 0; i < V; ++i)
                    cp_async4(dst + (p * 32 + lane) * V + i, base + p * t.plane_words + geom.col[i]);
            lr = lr + 1 == t.h ? 0 : lr + 1;
        }
        cp_async_commit();
    };
#pragma unroll
    for (int r = 0; r < DEPTH - 1; ++r) issue(r);

    auto step = [&](int st, auto parity) {
        constexpr int S = decltype(parity)::value;
        issue(st + DEPTH - 1);
        cp_async_wait<DEPTH - 1>();
        if (st < total) input_row<R, V>(smem + (st % DEPTH) * SLOT, lane, pend[0]);
        uint32_t out[V][P];
        skewed_step<R, K, V, S>(s, pend, out, geom.src_l, geom.src_r);
        const int j = st - 2 * K + 1;  // output sweep row
        if (j >= K && j < K + t.ny) strip_store<R, V>(t, geom, j - K, out);
    };
    for (int st = 0; st < steps; st += 2) {
        step(st, std::integral_constant<int, 0>{});
        if (st + 1 < steps) step(st + 1, std::integral_constant<int, 1>{});
    }
    cp_async_wait<0>();
}

} // namespace cb2
