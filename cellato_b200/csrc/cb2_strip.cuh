// cb2_strip.cuh -- the hot path's building blocks: a strip task and the
// register wavefront that advances one strip row through L generations.
//
// Work unit ("strip task"): a vertical strip of the grid.  Lane l of a warp
// holds V consecutive 32-bit words of every row, so a warp covers 32*V words:
// words 1 .. 32*V-2 of the segment are the strip's own columns and the two
// end words are its x halo.  The strip is swept top to bottom; each input row
// is read once (plus K halo rows above and below) and each output row is
// written once (cb2_pipe.cuh drives the sweep).
//
// Temporal blocking is a register wavefront: level g keeps the horizontal
// aggregates and centre states of its two most recent rows.  When a row of
// level g arrives, the row above it advances to level g+1 and is handed to
// level g+1 in the same pass, so one row pushed through L levels leaves as
// the row L rows further up, L generations later.
//
// Neighbours: left/right words come from the adjacent lanes through warp
// shuffles, and cells x-1 / x+1 are formed with funnel shifts across word
// boundaries.  Nothing is re-read from memory and nothing is wrapped with a
// modulo inside the loop; toroidal wrap (memory/interface.hpp:31-36) is
// folded into per-lane column indexes and the incremental row index.
//
// Halo correctness: a wrong value entering at either end word of the segment
// spreads one cell per generation, so for K <= 32 the strip's own words
// (segment words 1 .. 32V-2) are exact.  Rows are exact because the sweep
// starts K rows above and ends K rows below the strip's output rows.
#pragma once

#include <cstdint>
#include <type_traits>

#include "cb2_rules.cuh"

namespace cb2 {

// One warp's work: output rows [y0, y0+ny) of word columns [x0, x0+nx).
struct strip_task {
    const uint32_t* in;   // plane 0 of the source generation
    uint32_t* out;        // plane 0 of the destination generation
    int64_t plane_words;  // words per plane (wd * h)
    int32_t wd;           // 32-bit words per row
    int32_t h;            // rows
    int32_t x0, nx;       // first own word column, own word count (1 .. 32V-2)
    int32_t y0, ny;       // first output row, output row count (1 .. h - y0)
    int64_t t0;           // generation of the input (read by rules that depend on time)
    uint64_t seed;        // random seed of the run (read by stochastic rules)
    int64_t y_global0;    // global row of row 0 of these planes (a band's offset; 0 for a whole grid)
    int64_t global_h;     // rows of the whole grid (h for a whole grid)
};

// Where a lane's 32 cells are, for rules that read it (window rules): the
// generation the rule is evaluated at, the global row, the 32-bit word
// column (cells 32*xw .. 32*xw+31) and the run's seed.  Stochastic rules
// also get the level's lane keys (their random streams keyed up to the
// column, one per stream; null to key from scratch) and whether every lane
// of the warp shares its group of 64 cells with lane^1 in the same row
// (warp-uniform), in which case the pair splits the draws of that group.
struct cell_ctx {
    int64_t t;
    int64_t y;
    int64_t xw;
    uint64_t seed;
    const uint64_t* key = nullptr;
    bool paired = false;
    // The cells whose value of the node being evaluated is used; elsewhere
    // the node may return anything (a probability draw resolves only these).
    uint32_t care = 0xffffffffu;
};

// Where a row pushed into a level chain sits, for window rules (ast_rule):
// the generation of the chain's first level and the global row that level
// outputs (the row above its input); level g outputs the row g above that,
// modulo the grid's rows.
struct row_ctx {
    int64_t t;   // generation of the first level of the chain
    int64_t y;   // global row of the first level's output, 0 <= y < gh
    int64_t gh;  // rows of the whole grid
    uint64_t seed;
    bool paired;  // cell_ctx::paired
};

constexpr unsigned kFullMask = 0xffffffffu;

// What one lane of a warp works on within a strip task.
template <int V>
struct lane_geom {
    int64_t col[V];  // word column of each of the lane's words
    bool keep[V];    // the lane stores this word (one of the strip's own columns)
    int src_l;       // lane holding the word left of col[0]
    int src_r;       // lane holding the word right of col[V-1]
    int yoff;        // the lane's output rows start at t.y0 + yoff
    int rows;        // output rows the lane stores (<= t.ny)
};

// Strip geometry: the warp covers segment words x0-1 .. x0+32V-2 (mod wd);
// the two end words are halo, neighbours come from the adjacent lanes.
template <int V>
__device__ __forceinline__ lane_geom<V> strip_geom(const strip_task& t, int lane) {
    lane_geom<V> g;
#pragma unroll
    for (int i = 0; i < V; ++i) {
        const int off = V * lane + i;
        int c = (t.x0 - 1 + off) % t.wd;
        if (c < 0) c += t.wd;
        g.col[i] = c;
        g.keep[i] = off >= 1 && off <= t.nx;
    }
    g.src_l = lane > 0 ? lane - 1 : 0;
    g.src_r = lane < 31 ? lane + 1 : 31;
    g.yoff = 0;
    g.rows = t.ny;
    return g;
}

// Group geometry for narrow grids (wd <= 16 words, one word per lane): the
// warp holds `groups` copies of a whole row, each wd lanes wide, with exact
// toroidal wrap inside a group (no halo words); group q owns output rows
// t.y0 + q*t.ny .. + t.ny (clipped to the grid).  Lanes past the last group
// compute a duplicate of group 0's words and store nothing.
__device__ __forceinline__ lane_geom<1> group_geom(const strip_task& t, int groups, int lane) {
    lane_geom<1> g;
    const int wd = t.wd;
    int q = lane / wd, i = lane - q * wd;
    const bool live = q < groups;
    if (!live) q = 0;
    g.col[0] = i;
    g.src_l = q * wd + (i == 0 ? wd - 1 : i - 1);
    g.src_r = q * wd + (i == wd - 1 ? 0 : i + 1);
    g.yoff = q * t.ny;
    const int rows_left = t.h - (t.y0 + g.yoff);
    g.rows = live ? (rows_left < t.ny ? (rows_left > 0 ? rows_left : 0) : t.ny) : 0;
    g.keep[0] = live;
    return g;
}

// Banded geometry for a narrow strip (nx <= 14 own words, one word per lane):
// the warp holds `bands` side-by-side copies of the strip's segment, each
// nx + 2 lanes wide with a halo word at either end, and copy q sweeps output
// rows t.y0 + q*t.ny .. + t.ny of the same columns (clipped to the grid), so
// a narrow strip fills the warp instead of idling most of its lanes.  Lanes
// past the last copy compute a duplicate of copy 0's words and store nothing.
__device__ __forceinline__ lane_geom<1> band_geom(const strip_task& t, int bands, int lane) {
    lane_geom<1> g;
    const int s = t.nx + 2;
    int q = lane / s;
    const int i = lane - q * s;
    const bool live = q < bands;
    if (!live) q = 0;
    int c = (t.x0 - 1 + i) % t.wd;
    if (c < 0) c += t.wd;
    g.col[0] = c;
    g.src_l = q * s + (i > 0 ? i - 1 : 0);
    g.src_r = q * s + (i < s - 1 ? i + 1 : i);
    g.yoff = q * t.ny;
    const int rows_left = t.h - (t.y0 + g.yoff);
    g.rows = live ? (rows_left < t.ny ? (rows_left > 0 ? rows_left : 0) : t.ny) : 0;
    g.keep[0] = live && i >= 1 && i <= t.nx;
    return g;
}

// Per-level lane keys of a window rule that draws random numbers
// (R::level_keys); nothing for the other rules.
struct no_keys {
    static constexpr const uint64_t* k = nullptr;
};
template <class R, class = void>
struct keys_of {
    using type = no_keys;
};
template <class R>
struct keys_of<R, std::void_t<typename R::level_keys>> {
    using type = typename R::level_keys;
};
template <class R, class = void>
struct draws_of : std::false_type {};
template <class R>
struct draws_of<R, std::void_t<decltype(R::kDraws)>> : std::bool_constant<R::kDraws> {};
// Window rules that branch on the parity of the generation (R::kParity).
template <class R, class = void>
struct parity_of : std::false_type {};
template <class R>
struct parity_of<R, std::void_t<decltype(R::kParity)>> : std::bool_constant<R::kParity> {};

// Per-level row offsets of a window rule: level g outputs the row g above
// the first level's, and gm[g] = g mod (the grid's rows), so that one
// conditional add wraps it; nothing for the other rules.
template <int K>
struct level_rows {
    int64_t gm[K];
};
struct no_level_rows {};

template <class R, int K, int V>
struct strip_state {
    uint32_t h[K][2][V][R::NH];  // horizontal aggregates, slot = row parity
    uint32_t c[K][2][V][R::P];   // centre states, slot = row parity
    typename keys_of<R>::type keys[K][V];
    std::conditional_t<R::kWindow, level_rows<K>, no_level_rows> rows;
};

// One wavefront level: pushes `row` (a row of level g, parity slot Q) into
// the level's window and returns, in `row`, the row above it advanced one
// generation.
template <class R, int K, int V, int Q>
__device__ __forceinline__ void level_push(strip_state<R, K, V>& s, int g, uint32_t (&row)[V][R::P], int src_l,
                                           int src_r, const lane_geom<V>* geom = nullptr, const row_ctx* rc = nullptr) {
    constexpr int P = R::P, NH = R::NH;
    if constexpr (R::kWindow) {
        // window rule: (west, centre, east) word of every plane; the AST reads the
        // 3x3 window and the cells' generation and position
        uint32_t hc[V][NH];
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const uint32_t lw = __shfl_sync(kFullMask, row[V - 1][p], src_l);
            const uint32_t rw = __shfl_sync(kFullMask, row[0][p], src_r);
#pragma unroll
            for (int i = 0; i < V; ++i) {
                const uint32_t l = i == 0 ? lw : row[i - 1][p];
                const uint32_t r = i == V - 1 ? rw : row[i + 1][p];
                hc[i][3 * p] = west_of(l, row[i][p]);
                hc[i][3 * p + 1] = row[i][p];
                hc[i][3 * p + 2] = east_of(row[i][p], r);
            }
        }
        // level g outputs the row g above the first level's: no division and no
        // branch, which would split the unrolled levels' code
        int64_t y = rc->y - s.rows.gm[g];
        y = y < 0 ? y + rc->gh : y;
        uint32_t nxt[V][P];
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const cell_ctx c{rc->t + g, y, geom->col[i], rc->seed, s.keys[g][i].k, rc->paired};
            R::next_at(s.h[g][Q][i], s.h[g][1 - Q][i], hc[i], nxt[i], c);
        }
#pragma unroll
        for (int i = 0; i < V; ++i) {
#pragma unroll
            for (int k = 0; k < NH; ++k) s.h[g][Q][i][k] = hc[i][k];
#pragma unroll
            for (int p = 0; p < P; ++p) row[i][p] = nxt[i][p];
        }
    } else {
        uint32_t ind[V];
#pragma unroll
        for (int i = 0; i < V; ++i) ind[i] = R::indicator(row[i]);
        const uint32_t lw = __shfl_sync(kFullMask, ind[V - 1], src_l);
        const uint32_t rw = __shfl_sync(kFullMask, ind[0], src_r);
        uint32_t hc[V][NH];
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const uint32_t l = i == 0 ? lw : ind[i - 1];
            const uint32_t r = i == V - 1 ? rw : ind[i + 1];
            R::hagg(west_of(l, ind[i]), ind[i], east_of(ind[i], r), hc[i]);
        }
        uint32_t nxt[V][P];
#pragma unroll
        for (int i = 0; i < V; ++i) R::next(s.h[g][Q][i], s.h[g][1 - Q][i], hc[i], s.c[g][1 - Q][i], nxt[i]);
#pragma unroll
        for (int i = 0; i < V; ++i) {
#pragma unroll
            for (int k = 0; k < NH; ++k) s.h[g][Q][i][k] = hc[i][k];
#pragma unroll
            for (int p = 0; p < P; ++p) {
                s.c[g][Q][i][p] = row[i][p];
                row[i][p] = nxt[i][p];
            }
        }
    }
}

// Pushes one row through the K levels in sequence.  Q is the parity slot of
// this row; on return `row` holds the row K rows above it, advanced K
// generations.
template <class R, int K, int V, int Q>
__device__ __forceinline__ void strip_push(strip_state<R, K, V>& s, uint32_t (&row)[V][R::P], int src_l, int src_r,
                                           const lane_geom<V>* geom = nullptr, const row_ctx* rc = nullptr) {
#pragma unroll
    for (int g = 0; g < K; ++g) level_push<R, K, V, Q>(s, g, row, src_l, src_r, geom, rc);
}

// Two rows through one level, for rules that evaluate rows in pairs
// (has_pairs): `ra` has parity slot 0 and `rb` slot 1, so before the call slot
// 0 holds the aggregates of the row above ra's upper neighbour, slot 1 those
// of ra's upper neighbour (whose states are the centre c[1]).  The census rows
// shared by the two outputs -- ra's upper neighbour and ra -- are summed once
// (R::pair); each output adds its third row.  On return ra and rb hold the two
// rows above them advanced one generation, and the slots the same state as
// two level_push calls leave (c[0] is not kept: no pair push reads it).
template <class R, int K, int V>
__device__ __forceinline__ void level_push2(strip_state<R, K, V>& s, int g, uint32_t (&ra)[V][R::P],
                                            uint32_t (&rb)[V][R::P], int src_l, int src_r) {
    constexpr int P = R::P, NH = R::NH;
    uint32_t ia[V], ib[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
        ia[i] = R::indicator(ra[i]);
        ib[i] = R::indicator(rb[i]);
    }
    // the neighbour lanes' indicator words next to this lane's, for each row
    const uint32_t a_west = __shfl_sync(kFullMask, ia[V - 1], src_l);
    const uint32_t a_east = __shfl_sync(kFullMask, ia[0], src_r);
    const uint32_t b_west = __shfl_sync(kFullMask, ib[V - 1], src_l);
    const uint32_t b_east = __shfl_sync(kFullMask, ib[0], src_r);
    uint32_t ha[V][NH], hb[V][NH];
#pragma unroll
    for (int i = 0; i < V; ++i) {
        R::hagg(west_of(i == 0 ? a_west : ia[i - 1], ia[i]), ia[i], east_of(ia[i], i == V - 1 ? a_east : ia[i + 1]),
                ha[i]);
        R::hagg(west_of(i == 0 ? b_west : ib[i - 1], ib[i]), ib[i], east_of(ib[i], i == V - 1 ? b_east : ib[i + 1]),
                hb[i]);
    }
#pragma unroll
    for (int i = 0; i < V; ++i) {
        uint32_t q[3], oa[P], ob[P];
        R::pair(s.h[g][1][i], ha[i], q);
        R::next_pair(q, s.h[g][0][i], s.c[g][1][i], oa);
        R::next_pair(q, hb[i], ra[i], ob);
#pragma unroll
        for (int k = 0; k < NH; ++k) {
            s.h[g][0][i][k] = ha[i][k];
            s.h[g][1][i][k] = hb[i][k];
        }
#pragma unroll
        for (int p = 0; p < P; ++p) {
            s.c[g][1][i][p] = rb[i][p];
            ra[i][p] = oa[p];
            rb[i][p] = ob[p];
        }
    }
}

// Two consecutive rows (parity slots 0 and 1) through the K levels, level by
// level: the same result as strip_push<.., 0>(ra) then strip_push<.., 1>(rb).
template <class R, int K, int V>
__device__ __forceinline__ void strip_push2(strip_state<R, K, V>& s, uint32_t (&ra)[V][R::P], uint32_t (&rb)[V][R::P],
                                            int src_l, int src_r) {
#pragma unroll
    for (int g = 0; g < K; ++g) level_push2<R, K, V>(s, g, ra, rb, src_l, src_r);
}

// Skewed wavefront step: level g takes the row level g-1 produced in the
// previous step (held in pend[g]), so the K levels of one step are
// independent of each other.  pend[0] is the new input row; on return
// `out` holds the row leaving level K-1 and pend[g] the input of level g for
// the next step.  Level g receives row s - 2g at step s, so every level's
// rows alternate parity with the step parity S.
template <class R, int K, int V, int S>
__device__ __forceinline__ void skewed_step(strip_state<R, K, V>& s, uint32_t (&pend)[K][V][R::P],
                                            uint32_t (&out)[V][R::P], int src_l, int src_r) {
#pragma unroll
    for (int g = 0; g < K; ++g) level_push<R, K, V, S>(s, g, pend[g], src_l, src_r);
#pragma unroll
    for (int i = 0; i < V; ++i)
#pragma unroll
        for (int p = 0; p < R::P; ++p) out[i][p] = pend[K - 1][i][p];
#pragma unroll
    for (int g = K - 1; g > 0; --g)
#pragma unroll
        for (int i = 0; i < V; ++i)
#pragma unroll
            for (int p = 0; p < R::P; ++p) pend[g][i][p] = pend[g - 1][i][p];
}

// Stores the lane's words of output row t.y0 + geom.yoff + j (0 <= j < geom.rows),
// back in dictionary indexes (decode_states).
template <class R, int V>
__device__ __forceinline__ void strip_store(const strip_task& t, const lane_geom<V>& geom, int j,
                                            const uint32_t (&src)[V][R::P]) {
    if (j >= geom.rows) return;
    uint32_t* base = t.out + (int64_t)(t.y0 + geom.yoff + j) * t.wd;
    uint32_t w[V][R::P];
#pragma unroll
    for (int i = 0; i < V; ++i) {
#pragma unroll
        for (int p = 0; p < R::P; ++p) w[i][p] = src[i][p];
        decode_states<R>(w[i]);
    }
#pragma unroll
    for (int p = 0; p < R::P; ++p)
#pragma unroll
        for (int i = 0; i < V; ++i)
            if (geom.keep[i]) base[p * t.plane_words + geom.col[i]] = w[i][p];
}

} // namespace cb2
