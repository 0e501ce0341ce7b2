// cb2_api.cpp -- implementation of the C-ABI in include/cellato_b200.h:
// automaton registry, owning device grids, layout upload/download, run
// planning (temporal depth, lane width, strip height), the autotuner and the
// measurement helpers.
#include "cellato_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "cb2_internal.h"

namespace cb2 {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

static int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

static int cuda_fail(cudaError_t e, const char* what) {
    return fail(CB2_ECUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define CB2_CUDA(call)                                                                                                 \
    do {                                                                                                               \
        cudaError_t e_ = (call);                                                                                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);                                                            \
    } while (0)

// The hand-written networks (cb2_rules.cuh).  Their dictionaries list the
// states in enum order (game_of_life/config.hpp:21, wire/config.hpp:21-24,
// excitable/config.hpp:21-28), so index and state value coincide.
static const int64_t kIdentity[32] = {0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15,
                                      16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31};
static const automaton_desc kBuiltin[kNumBuiltin] = {
    {"game-of-life", 1, 2, kIdentity}, {"wire", 2, 4, kIdentity}, {"excitable", 3, 8, kIdentity}};

int automaton_count() { return kNumBuiltin + generic_count(); }

const automaton_desc* automaton_at(int id) {
    if (id >= 0 && id < kNumBuiltin) return &kBuiltin[id];
    if (id >= kNumBuiltin && id < automaton_count()) return generic_desc(id - kNumBuiltin);
    return nullptr;
}

int planes_of(int automaton) {
    const automaton_desc* d = automaton_at(automaton);
    return d ? d->planes : -1;
}

const char* name_of(int automaton) {
    const automaton_desc* d = automaton_at(automaton);
    return d ? d->name : nullptr;
}

int find_automaton(const char* name) {
    if (!name) return -1;
    for (int i = 0; i < automaton_count(); ++i)
        if (std::strcmp(name, name_of(i)) == 0) return i;
    return -1;
}

// ---- tuning table -----------------------------------------------------------

struct tune_key {
    int automaton;
    int64_t x, y;
    bool operator<(const tune_key& o) const { return std::tie(automaton, x, y) < std::tie(o.automaton, o.x, o.y); }
};

static std::mutex g_tune_mu;
static std::map<tune_key, cb2_tuning> g_tune;

static int log2_floor(int64_t v) {
    int l = 0;
    while (v > 1) {
        v >>= 1;
        ++l;
    }
    return l;
}

// Exact size first, then the nearest entry in the same power-of-two bucket.
static bool tuned_entry(int automaton, int64_t x, int64_t y, cb2_tuning* out) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find({automaton, x, y});
    if (it != g_tune.end()) {
        *out = it->second;
        return true;
    }
    for (auto& kv : g_tune)
        if (kv.first.automaton == automaton && log2_floor(kv.first.x) == log2_floor(x) &&
            log2_floor(kv.first.y) == log2_floor(y)) {
            *out = kv.second;
            return true;
        }
    return false;
}

static bool valid_k(int k) { return k == 1 || k == 2 || k == 4 || k == 8 || k == 16 || k == 32; }

// Default (K, V, L, rows per step) per automaton, the fastest plans measured
// on B200 at the headline sizes; cb2_autotune replaces them per size.
// Two warps per CTA for all three: at the headline sizes the autotuner
// prefers one-warp CTAs for WireWorld (K32 V1 L32) and Greenberg-Hastings
// (K16 V2 L16) by a few per cent, but on small grids a single warp's chain of
// 16 or 32 levels serialises each task (requests of sides 128..16384 one at a
// time: 1.70 against 1.98 Tcell/s), so the defaults stay the shapes that hold
// up across sizes.
static const int kDefaultPlan[kNumBuiltin][4] = {{32, 2, 16, 4}, {16, 2, 8, 4}, {32, 2, 16, 4}};
// Lowered DSL automata: a window of 3P words per row and level keeps the
// register count in check only for short chains.
static const int kDefaultDslPlan[4] = {8, 1, 2, 2};
// The bundled lowered automata and the two stochastic examples: the plans
// cb2_autotune picked for each at 16384^2 with uniform states (most go
// sixteen levels deep; the Margolus, two-draw and 32-state ones stay short).
struct named_plan {
    const char* name;
    int plan[4];
};
static const named_plan kMeasuredDslPlans[] = {
    {"brian", {16, 1, 4, 2}},    {"forest-fire", {16, 1, 4, 2}}, {"fluid", {16, 1, 4, 2}},
    {"maze", {16, 1, 4, 2}},     {"traffic", {16, 1, 4, 2}},     {"critters", {8, 2, 2, 2}},
    {"noisy-life", {16, 1, 4, 2}}, {"cyclic", {8, 1, 4, 2}},     {"lightning-forest", {4, 1, 1, 2}},
};

static const int* default_plan(int automaton) {
    if (automaton < kNumBuiltin) return kDefaultPlan[automaton];
    const char* name = name_of(automaton);
    for (const named_plan& p : kMeasuredDslPlans)
        if (name && std::strcmp(name, p.name) == 0 && find_variant(automaton, p.plan[0], p.plan[1], p.plan[2], p.plan[3]))
            return p.plan;
    return kDefaultDslPlan;
}

// Fills every 0 field of `t` for a grid of geometry g.
int resolve_plan(const grid_geom& g, const cb2_tuning* t, run_plan* plan) {
    cb2_tuning want{0, 0, 0, 0, 0};
    if (t) want = *t;
    cb2_tuning tuned{0, 0, 0, 0, 0};
    const bool have_tuned = tuned_entry(g.automaton, g.x_size, g.y_size, &tuned);
    const int* def = default_plan(g.automaton);
    const int k = want.temporal_steps ? want.temporal_steps : (have_tuned ? tuned.temporal_steps : def[0]);
    if (!valid_k(k))
        return fail(CB2_EINVAL, "temporal_steps must be 1, 2, 4, 8, 16 or 32 (got " + std::to_string(k) + ")");
    const bool tuned_k = have_tuned && tuned.temporal_steps == k;
    int v = want.words_per_lane;
    if (!v) {
        v = tuned_k ? tuned.words_per_lane : (g.wd <= 30 ? 1 : (k == def[0] ? def[1] : 2));
        if (!find_variant(g.automaton, k, v, 0)) {  // the automaton's table has no kernel that wide at this K
            const strip_variant* any = find_variant(g.automaton, k, 0, 0);
            if (any) v = any->v;
        }
    }
    if (v != 1 && v != 2 && v != 4)
        return fail(CB2_EINVAL, "words_per_lane must be 1, 2 or 4 (got " + std::to_string(v) + ")");
    int l = want.levels_per_warp;
    if (!l) l = (tuned_k && tuned.words_per_lane == v) ? tuned.levels_per_warp : (k == def[0] && v == def[1] ? def[2] : 0);
    int r = want.rows_per_step;
    if (r && r != 1 && r != 2 && r != 4)
        return fail(CB2_EINVAL, "rows_per_step must be 1, 2 or 4 (got " + std::to_string(r) + ")");
    if (!r)
        r = (tuned_k && tuned.words_per_lane == v && tuned.levels_per_warp == l)
                ? tuned.rows_per_step
                : (k == def[0] && v == def[1] && l == def[2] ? def[3] : 0);
    const strip_variant* sv = find_variant(g.automaton, k, v, l, r);
    if (!sv && !want.levels_per_warp && !want.rows_per_step) sv = find_variant(g.automaton, k, v, 0);
    if (!sv)
        return fail(CB2_EINVAL, "no strip kernel for temporal_steps=" + std::to_string(k) + ", words_per_lane=" +
                                    std::to_string(v) + ", levels_per_warp=" + std::to_string(l) +
                                    ", rows_per_step=" + std::to_string(r));
    int rows = want.tile_rows;
    if (!rows && tuned_k && tuned.words_per_lane == sv->v && tuned.levels_per_warp == sv->l &&
        tuned.rows_per_step == sv->r)
        rows = tuned.tile_rows;
    if (!rows) rows = auto_tile_rows(g, *sv);
    if (rows < 1) return fail(CB2_EINVAL, "tile_rows must be positive");
    plan->k = sv->k;
    plan->v = sv->v;
    plan->l = sv->l;
    plan->r = sv->r;
    plan->tile_rows = std::min(rows, (int)g.h);
    return CB2_OK;
}

int make_geom(int automaton, int64_t x, int64_t y, grid_geom* g) {
    const int P = planes_of(automaton);
    if (P < 0) return fail(CB2_ENOTFOUND, "unknown automaton id " + std::to_string(automaton));
    if (x <= 0 || y <= 0) return fail(CB2_EINVAL, "grid sizes must be positive");
    if (x % 32) return fail(CB2_EINVAL, "x_size must be a multiple of 32 (got " + std::to_string(x) + ")");
    if (x / 32 > (1 << 30) || y > (1 << 30)) return fail(CB2_EINVAL, "grid too large");
    g->automaton = automaton;
    g->planes = P;
    g->states = automaton_at(automaton)->states;
    g->x_size = x;
    g->y_size = y;
    g->wd = (int32_t)(x / 32);
    g->h = (int32_t)y;
    g->plane_words = (int64_t)g->wd * g->h;
    return CB2_OK;
}

// Launches `steps` generations from `cur` (buffer index) alternating with
// the other buffer; returns the index that holds the result.
int run_chunks(const grid_geom& g, uint32_t* const bufs[2], int cur, int64_t steps, const cb2_tuning* tuning,
               cudaStream_t stream, int* result, int64_t t0, uint64_t seed) {
    run_plan main_plan;
    int rc = resolve_plan(g, tuning, &main_plan);
    if (rc) return rc;
    int64_t left = steps;
    while (left > 0) {
        run_plan p = main_plan;
        if (left < p.k) {  // remainder in powers of two, same lane width where possible
            int k = 1;
            while (k * 2 <= left) k *= 2;
            cb2_tuning t2{k, 0, p.v, 0, 0};
            if (!find_variant(g.automaton, k, p.v, 0)) t2.words_per_lane = 0;
            rc = resolve_plan(g, &t2, &p);
            if (rc) return rc;
        }
        cudaError_t e = launch_strip_pass(g, bufs[cur], bufs[1 - cur], p, stream, t0 + (steps - left), seed);
        if (e != cudaSuccess) return cuda_fail(e, "strip kernel launch");
        cur = 1 - cur;
        left -= p.k;
    }
    *result = cur;
    return CB2_OK;
}

} // namespace cb2

using namespace cb2;


extern "C" {

int cb2_abi_version(void) { return CB2_ABI_VERSION; }

const char* cb2_last_error(void) { return g_last_error.c_str(); }

int cb2_automaton_lookup(const char* name) {
    const int id = find_automaton(name);
    if (id < 0) return fail(CB2_ENOTFOUND, std::string("unknown automaton '") + (name ? name : "(null)") + "'");
    return id;
}

int cb2_automaton_info(int id, const char** name, int* planes, int* states) {
    const automaton_desc* d = automaton_at(id);
    if (!d) return fail(CB2_ENOTFOUND, "unknown automaton id " + std::to_string(id));
    if (name) *name = d->name;
    if (planes) *planes = d->planes;
    if (states) *states = d->states;
    return CB2_OK;
}

int cb2_automaton_count(void) { return automaton_count(); }

int cb2_automaton_fingerprint(int id, uint64_t* fingerprint) {
    const automaton_desc* d = automaton_at(id);
    if (!d) return fail(CB2_ENOTFOUND, "unknown automaton id " + std::to_string(id));
    if (!fingerprint) return fail(CB2_EINVAL, "null output");
    const uint64_t fp = id < kNumBuiltin ? builtin_fingerprint(id) : d->fingerprint;
    if (!fp)
        return fail(CB2_ENOTFOUND, "the library was built without the Cellato headers and cannot tell which rule "
                                   "automaton '" + std::string(d->name) + "' is");
    *fingerprint = fp;
    return CB2_OK;
}

int cb2_automaton_values(int id, int64_t* values, int capacity) {
    const automaton_desc* d = automaton_at(id);
    if (!d) return fail(CB2_ENOTFOUND, "unknown automaton id " + std::to_string(id));
    for (int i = 0; values && i < capacity && i < d->states; ++i) values[i] = d->values[i];
    return d->states;
}

int64_t cb2_layout_bytes(int automaton, int layout, int word_bits, int64_t x, int64_t y) {
    const int P = planes_of(automaton);
    if (P < 0) return fail(CB2_ENOTFOUND, "unknown automaton id " + std::to_string(automaton));
    if (x <= 0 || y <= 0) return fail(CB2_EINVAL, "grid sizes must be positive");
    switch (layout) {
    case CB2_LAYOUT_STANDARD:
        if (word_bits != 8 && word_bits != 32) return fail(CB2_EINVAL, "standard cells are 8 or 32 bits");
        return x * y * (word_bits / 8);
    case CB2_LAYOUT_BIT_PLANES:
        if (word_bits != 32 && word_bits != 64) return fail(CB2_EINVAL, "word_bits must be 32 or 64");
        if (x % word_bits) return fail(CB2_EINVAL, "`x_size` must be a multiple of `word store bits`");
        return (int64_t)P * y * (x / 8);
    case CB2_LAYOUT_BIT_ARRAY: {
        if (word_bits != 32 && word_bits != 64) return fail(CB2_EINVAL, "word_bits must be 32 or 64");
        const int cpw = word_bits / P;
        if (x % cpw)
            return fail(CB2_EINVAL, "Grid x_size must be divisible by cells_per_word. x_size=" + std::to_string(x) +
                                        ", cells_per_word=" + std::to_string(cpw));
        return x * y / cpw * (word_bits / 8);
    }
    case CB2_LAYOUT_TILED_BIT_PLANES: {
        if (word_bits != 32 && word_bits != 64) return fail(CB2_EINVAL, "word_bits must be 32 or 64");
        if (x % 8 || y % (word_bits / 8))
            return fail(CB2_EINVAL, "`x_size` and `y_size` must be multiples of `x_word_tile_size` and "
                                    "`y_word_tile_size`");
        return (int64_t)P * x * y / 8;
    }
    default: return fail(CB2_EINVAL, "unknown layout " + std::to_string(layout));
    }
}

int cb2_run_bit_planes(int automaton, void* const* a, void* const* b, int64_t x_size, int64_t y_size, int64_t steps,
                       const cb2_tuning* tuning, void* stream, int* result_in_b) {
    return cb2_run_bit_planes_at(automaton, a, b, x_size, y_size, 0, steps, kDefaultSeed, tuning, stream, result_in_b);
}

int cb2_run_bit_planes_at(int automaton, void* const* a, void* const* b, int64_t x_size, int64_t y_size,
                          int64_t time_step, int64_t steps, uint64_t seed, const cb2_tuning* tuning, void* stream,
                          int* result_in_b) {
    grid_geom g;
    int rc = make_geom(automaton, x_size, y_size, &g);
    if (rc) return rc;
    if (!a || !b || steps < 0) return fail(CB2_EINVAL, "null plane array or negative steps");
    // The kernel addresses plane p at plane0 + p * plane_words: the caller's
    // planes must be one allocation at that stride.
    for (int p = 1; p < g.planes; ++p) {
        if ((char*)a[p] - (char*)a[0] != (ptrdiff_t)(p * g.plane_words * 4) ||
            (char*)b[p] - (char*)b[0] != (ptrdiff_t)(p * g.plane_words * 4))
            return fail(CB2_EINVAL, "planes must be consecutive in one allocation (stride = y_size * x_size / 8 bytes)");
    }
    if (time_step < 0) return fail(CB2_EINVAL, "time_step must be non-negative");
    uint32_t* const bufs[2] = {(uint32_t*)a[0], (uint32_t*)b[0]};
    int res = 0;
    rc = run_chunks(g, bufs, 0, steps, tuning, (cudaStream_t)stream, &res, time_step, seed);
    if (rc) return rc;
    if (result_in_b) *result_in_b = res;
    return CB2_OK;
}

int cb2_grid_create(int automaton, int64_t x_size, int64_t y_size, cb2_grid** out) {
    if (!out) return fail(CB2_EINVAL, "null output pointer");
    grid_geom g;
    int rc = make_geom(automaton, x_size, y_size, &g);
    if (rc) return rc;
    cb2_grid* grid = new cb2_grid();
    grid->g = g;
    cudaGetDevice(&grid->device);
    const size_t bytes = (size_t)g.planes * g.plane_words * 4;
    cudaError_t e = cudaMalloc(&grid->buf[0], bytes);
    if (e == cudaSuccess) e = cudaMalloc(&grid->buf[1], bytes);
    if (e == cudaSuccess) e = cudaMalloc(&grid->flag, sizeof(unsigned) + 16 * sizeof(unsigned long long) + 12);
    if (e == cudaSuccess) e = cudaMemset(grid->buf[0], 0, bytes);
    if (e != cudaSuccess) {
        cb2_grid_destroy(grid);
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? CB2_ENOMEM : CB2_ECUDA,
                    std::string("grid allocation: ") + cudaGetErrorString(e));
    }
    grid->sums = (unsigned long long*)((char*)grid->flag + 16);
    *out = grid;
    return CB2_OK;
}

int cb2_grid_destroy(cb2_grid* grid) {
    if (!grid) return CB2_OK;
    cudaFree(grid->buf[0]);
    cudaFree(grid->buf[1]);
    cudaFree(grid->staging);
    cudaFree(grid->flag);
    delete grid;
    return CB2_OK;
}

static int ensure_staging(cb2_grid* grid, size_t bytes) {
    if (grid->staging_bytes >= bytes) return CB2_OK;
    cudaFree(grid->staging);
    grid->staging = nullptr;
    grid->staging_bytes = 0;
    cudaError_t e = cudaMalloc(&grid->staging, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(CB2_ENOMEM, std::string("staging allocation: ") + cudaGetErrorString(e));
    }
    grid->staging_bytes = bytes;
    return CB2_OK;
}

// Enqueues the upload of a host image (copy, and the layout conversion) on s.
static int enqueue_upload(cb2_grid* grid, int layout, int word_bits, const void* host, size_t bytes, cudaStream_t s) {
    if (!grid || !host) return fail(CB2_EINVAL, "null grid or host pointer");
    const grid_geom& g = grid->g;
    const int64_t need = cb2_layout_bytes(g.automaton, layout, word_bits, g.x_size, g.y_size);
    if (need < 0) return (int)need;
    if ((int64_t)bytes != need)
        return fail(CB2_EINVAL, "host image is " + std::to_string(bytes) + " bytes, layout needs " + std::to_string(need));
    uint32_t* dst = grid->buf[grid->cur];
    if (layout == CB2_LAYOUT_BIT_PLANES ||
        (layout == CB2_LAYOUT_BIT_ARRAY && g.planes == 1)) {  // one plane: bit_array == bit_planes bytes
        CB2_CUDA(cudaMemcpyAsync(dst, host, bytes, cudaMemcpyHostToDevice, s));
    } else {
        int rc = ensure_staging(grid, bytes);
        if (rc) return rc;
        CB2_CUDA(cudaMemcpyAsync(grid->staging, host, bytes, cudaMemcpyHostToDevice, s));
        cudaError_t e = cudaSuccess;
        if (layout == CB2_LAYOUT_STANDARD) {
            CB2_CUDA(cudaMemsetAsync(grid->flag, 0, sizeof(unsigned), s));
            e = launch_pack_cells(g, grid->staging, word_bits / 8, dst, grid->flag, s);
        } else if (layout == CB2_LAYOUT_BIT_ARRAY) {
            e = launch_bit_array_to_planes(g, grid->staging, word_bits, dst, s);
        } else {
            e = launch_tiled_to_planes(g, grid->staging, word_bits, dst, s);
        }
        if (e != cudaSuccess) return cuda_fail(e, "layout conversion launch");
    }
    grid->time_step = 0;
    return CB2_OK;
}

int cb2_grid_upload(cb2_grid* grid, int layout, int word_bits, const void* host, size_t bytes, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    int rc = enqueue_upload(grid, layout, word_bits, host, bytes, s);
    if (rc) return rc;
    CB2_CUDA(cudaStreamSynchronize(s));
    if (layout == CB2_LAYOUT_STANDARD) {
        unsigned bad = 0;
        CB2_CUDA(cudaMemcpy(&bad, grid->flag, sizeof(unsigned), cudaMemcpyDeviceToHost));
        if (bad) return fail(CB2_ESTATE, "State not found in dictionary (a cell value exceeds the automaton's states)");
    }
    return CB2_OK;
}

int cb2_grid_upload_async(cb2_grid* grid, int layout, int word_bits, const void* host, size_t bytes, void* stream) {
    if (layout == CB2_LAYOUT_STANDARD)
        return fail(CB2_EINVAL, "the standard layout's cells are checked on the host: use cb2_grid_upload");
    return enqueue_upload(grid, layout, word_bits, host, bytes, (cudaStream_t)stream);
}

// Enqueues the download of the current generation (conversion, and copy) on s.
static int enqueue_download(cb2_grid* grid, int layout, int word_bits, void* host, size_t bytes, cudaStream_t s) {
    if (!grid || !host) return fail(CB2_EINVAL, "null grid or host pointer");
    const grid_geom& g = grid->g;
    const int64_t need = cb2_layout_bytes(g.automaton, layout, word_bits, g.x_size, g.y_size);
    if (need < 0) return (int)need;
    if ((int64_t)bytes != need)
        return fail(CB2_EINVAL, "host image is " + std::to_string(bytes) + " bytes, layout needs " + std::to_string(need));
    const uint32_t* src = grid->buf[grid->cur];
    if (layout == CB2_LAYOUT_BIT_PLANES || (layout == CB2_LAYOUT_BIT_ARRAY && g.planes == 1)) {
        CB2_CUDA(cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, s));
    } else {
        int rc = ensure_staging(grid, bytes);
        if (rc) return rc;
        cudaError_t e = cudaSuccess;
        if (layout == CB2_LAYOUT_STANDARD)
            e = launch_unpack_cells(g, src, grid->staging, word_bits / 8, s);
        else if (layout == CB2_LAYOUT_BIT_ARRAY)
            e = launch_planes_to_bit_array(g, src, grid->staging, word_bits, s);
        else
            e = launch_planes_to_tiled(g, src, grid->staging, word_bits, s);
        if (e != cudaSuccess) return cuda_fail(e, "layout conversion launch");
        CB2_CUDA(cudaMemcpyAsync(host, grid->staging, bytes, cudaMemcpyDeviceToHost, s));
    }
    return CB2_OK;
}

int cb2_grid_download(cb2_grid* grid, int layout, int word_bits, void* host, size_t bytes, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    int rc = enqueue_download(grid, layout, word_bits, host, bytes, s);
    if (rc) return rc;
    CB2_CUDA(cudaStreamSynchronize(s));
    return CB2_OK;
}

int cb2_grid_download_async(cb2_grid* grid, int layout, int word_bits, void* host, size_t bytes, void* stream) {
    return enqueue_download(grid, layout, word_bits, host, bytes, (cudaStream_t)stream);
}

int cb2_grid_fill_random(cb2_grid* grid, uint64_t seed, const uint64_t* thresholds, int n, void* stream) {
    if (!grid) return fail(CB2_EINVAL, "null grid");
    if (n < 0 || n > kMaxThresholds || (n && !thresholds))
        return fail(CB2_EINVAL, "between 0 and " + std::to_string(kMaxThresholds) + " thresholds are supported");
    if (n >= grid->g.states) return fail(CB2_EINVAL, "more thresholds than the automaton has states - 1");
    for (int i = 1; i < n; ++i)
        if (thresholds[i] < thresholds[i - 1]) return fail(CB2_EINVAL, "thresholds must be non-decreasing");
    cudaError_t e = launch_fill_random(grid->g, grid->buf[grid->cur], seed, thresholds, n, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "fill_random launch");
    grid->time_step = 0;
    return CB2_OK;
}

int cb2_grid_run(cb2_grid* grid, int64_t steps, const cb2_tuning* tuning, void* stream) {
    if (!grid) return fail(CB2_EINVAL, "null grid");
    if (steps < 0) return fail(CB2_EINVAL, "steps must be non-negative");
    int res = grid->cur;
    int rc = run_chunks(grid->g, grid->buf, grid->cur, steps, tuning, (cudaStream_t)stream, &res, grid->time_step,
                        grid->seed);
    if (rc) return rc;
    grid->cur = res;
    grid->time_step += steps;
    return CB2_OK;
}

int cb2_grid_set_seed(cb2_grid* grid, uint64_t seed) {
    if (!grid) return fail(CB2_EINVAL, "null grid");
    grid->seed = seed;
    return CB2_OK;
}

int cb2_grid_set_time_step(cb2_grid* grid, int64_t time_step) {
    if (!grid || time_step < 0) return fail(CB2_EINVAL, "null grid or negative time_step");
    grid->time_step = time_step;
    return CB2_OK;
}

int cb2_grid_checksum(cb2_grid* grid, const int64_t* values, int n_values, uint64_t out[16], void* stream) {
    if (!grid || !out) return fail(CB2_EINVAL, "null grid or output");
    if (n_values < 0 || n_values > (1 << kMaxPlanes) || (n_values && !values))
        return fail(CB2_EINVAL, "state_values must hold at most " + std::to_string(1 << kMaxPlanes) + " entries");
    if (!values) {  // the dictionary's own state values, as the reference's standard grid sums them
        const automaton_desc* d = automaton_at(grid->g.automaton);
        values = d->values;
        n_values = d->states;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CB2_CUDA(cudaMemsetAsync(grid->sums, 0, 16 * sizeof(unsigned long long), s));
    cudaError_t e = launch_checksum(grid->g, grid->buf[grid->cur], values, n_values, grid->sums, s);
    if (e != cudaSuccess) return cuda_fail(e, "checksum launch");
    unsigned long long host[16];
    CB2_CUDA(cudaMemcpyAsync(host, grid->sums, sizeof(host), cudaMemcpyDeviceToHost, s));
    CB2_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < 16; ++i) out[i] = host[i];
    return CB2_OK;
}

int cb2_grid_planes(cb2_grid* grid, void** planes, int* n_planes, int64_t* words_per_plane) {
    if (!grid) return fail(CB2_EINVAL, "null grid");
    if (planes)
        for (int p = 0; p < grid->g.planes; ++p) planes[p] = grid->buf[grid->cur] + p * grid->g.plane_words;
    if (n_planes) *n_planes = grid->g.planes;
    if (words_per_plane) *words_per_plane = grid->g.plane_words;
    return CB2_OK;
}

int64_t cb2_grid_time_step(const cb2_grid* grid) { return grid ? grid->time_step : -1; }

int cb2_plan(int automaton, int64_t x_size, int64_t y_size, const cb2_tuning* tuning, cb2_tuning* plan) {
    grid_geom g;
    int rc = make_geom(automaton, x_size, y_size, &g);
    if (rc) return rc;
    run_plan p;
    rc = resolve_plan(g, tuning, &p);
    if (rc) return rc;
    if (plan) *plan = cb2_tuning{p.k, p.tile_rows, p.v, p.l, p.r};
    return CB2_OK;
}

int cb2_variants(int automaton, cb2_tuning* out, int capacity) {
    if (planes_of(automaton) < 0) return fail(CB2_ENOTFOUND, "unknown automaton id " + std::to_string(automaton));
    const std::vector<strip_variant>& vs = strip_variants(automaton);
    for (int i = 0; out && i < capacity && i < (int)vs.size(); ++i)
        out[i] = cb2_tuning{vs[i].k, 0, vs[i].v, vs[i].l, vs[i].r};
    return (int)vs.size();
}

int cb2_autotune(int automaton, int64_t x_size, int64_t y_size, double budget_ms, cb2_tuning* best) {
    grid_geom g;
    int rc = make_geom(automaton, x_size, y_size, &g);
    if (rc) return rc;
    if (budget_ms <= 0) budget_ms = 20000;
    cb2_grid* grid = nullptr;
    rc = cb2_grid_create(automaton, x_size, y_size, &grid);
    if (rc) return rc;
    // uniform states: thresholds j * 2^53 / states for j = 1 .. states - 1
    uint64_t thr[kMaxThresholds];
    for (int j = 1; j < g.states; ++j) thr[j - 1] = (uint64_t)(((unsigned __int128)j << 53) / (unsigned)g.states);
    rc = cb2_grid_fill_random(grid, 1, thr, g.states - 1, nullptr);
    if (rc) {
        cb2_grid_destroy(grid);
        return rc;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<cb2_tuning> cands;
    for (const strip_variant& sv : strip_variants(automaton)) {
        if (sv.k < 4) continue;  // one- and two-generation passes are memory-bound at any size
        const int rows = auto_tile_rows(g, sv);
        cands.push_back(cb2_tuning{sv.k, rows, sv.v, sv.l, sv.r});
        if (rows * 2 <= (int)g.h) cands.push_back(cb2_tuning{sv.k, rows * 2, sv.v, sv.l, sv.r});
    }
    double best_ns = 1e300;
    cb2_tuning pick = cands.front();
    double spent = 0;
    for (const cb2_tuning& c : cands) {
        if (spent > budget_ms) break;
        const int64_t gens = 32;  // the same generations for every candidate
        rc = cb2_grid_run(grid, c.temporal_steps, &c, nullptr);  // warm-up
        if (rc) break;
        cudaEventRecord(e0);
        rc = cb2_grid_run(grid, gens, &c, nullptr);
        if (rc) break;
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        spent += ms * 1.5;
        const double ns_per_gen = ms * 1e6 / gens;
        if (ns_per_gen < best_ns) {
            best_ns = ns_per_gen;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cb2_grid_destroy(grid);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune[{automaton, x_size, y_size}] = pick;
    }
    if (best) *best = pick;
    return CB2_OK;
}

int cb2_tuning_load(const char* path) {
    std::ifstream f(path ? path : "");
    if (!f) return fail(CB2_ENOTFOUND, std::string("cannot open tuning file ") + (path ? path : "(null)"));
    std::string line;
    int n = 0;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream is(line);
        std::string name;
        long long x, y;
        cb2_tuning t{};
        if (!(is >> name >> x >> y >> t.temporal_steps >> t.tile_rows >> t.words_per_lane >> t.levels_per_warp))
            return fail(CB2_EINVAL, "malformed tuning line: " + line);
        if (!(is >> t.rows_per_step)) t.rows_per_step = 1;  // lines written before the field existed
        int a = find_automaton(name.c_str());
        if (a < 0) return fail(CB2_ENOTFOUND, "unknown automaton in tuning file: " + name);
        if (!valid_k(t.temporal_steps) ||
            !find_variant(a, t.temporal_steps, t.words_per_lane, t.levels_per_warp, t.rows_per_step) ||
            t.tile_rows < 1)
            return fail(CB2_EINVAL, "invalid tuning values: " + line);
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune[{a, x, y}] = t;
        ++n;
    }
    return n;
}

int cb2_tuning_save(const char* path) {
    std::ofstream f(path ? path : "");
    if (!f) return fail(CB2_EINVAL, std::string("cannot write tuning file ") + (path ? path : "(null)"));
    f << "# automaton x_size y_size temporal_steps tile_rows words_per_lane levels_per_warp rows_per_step\n";
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (auto& kv : g_tune)
        f << name_of(kv.first.automaton) << ' ' << kv.first.x << ' ' << kv.first.y << ' ' << kv.second.temporal_steps
          << ' ' << kv.second.tile_rows << ' ' << kv.second.words_per_lane << ' ' << kv.second.levels_per_warp
          << ' ' << kv.second.rows_per_step << '\n';
    return (int)g_tune.size();
}

int cb2_measure_lop3_peak(double* ops_per_second) {
    if (!ops_per_second) return fail(CB2_EINVAL, "null output");
    int dev = 0, sms = 0;
    CB2_CUDA(cudaGetDevice(&dev));
    CB2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint32_t* sink = nullptr;
    CB2_CUDA(cudaMalloc(&sink, 4));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 256, blocks = sms * 8, iters = 4096;
    double best = 0;
    cudaError_t e = cudaSuccess;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
        cudaEventRecord(e0);
        e = launch_lop3_probe(sink, blocks, threads, iters, nullptr);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = (double)blocks * threads * iters * kLop3ProbeOpsPerIter;
        if (rep > 0 && ms > 0) best = std::max(best, ops / (ms * 1e-3));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(e, "lop3 probe");
    *ops_per_second = best;
    return CB2_OK;
}

int cb2_network_ops(int automaton, double* alu, double* shuffles) {
    // Per 32-bit word per generation (cb2_rules.cuh): two funnel shifts for
    // the west/east neighbour words, plus the rule's logic ops with rows
    // evaluated in pairs -- every plan of two or more rows per step -- (game
    // of life 9, 10 row by row; wireworld 8, 10 row by row;
    // greenberg-hastings 5 three-input operations on its shift-register
    // encoding); two shuffles per lane per row, shared by the lane's V = 2
    // words.
    static const double kLogic[kNumBuiltin] = {9, 8, 5};
    if (automaton >= kNumBuiltin && automaton < automaton_count())
        return fail(CB2_EINVAL, "no static operation count for a lowered DSL automaton");
    if (automaton < 0 || automaton >= kNumBuiltin) return fail(CB2_ENOTFOUND, "unknown automaton");
    if (alu) *alu = kLogic[automaton] + 2;
    if (shuffles) *shuffles = 1.0;
    return CB2_OK;
}

} // extern "C"
