// cb2_kernels.cu -- device kernels of the library and their launchers.
//
//  * pipe_kernel<Rule, K, V, L, RPS> the hot path (cb2_pipe.cuh), K
//                               generations per launch over a whole grid
//  * layout conversion kernels  standard / bit_array / tiled host images to
//                               and from the device's linear bit planes
//  * fill_random_kernel         the seeded SplitMix64 input generator
//  * checksum_kernel            the reference's 16-tile checksum from planes
//  * lop3_probe_kernel          integer-pipe peak probe for the roofline
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include "cb2_internal.h"
#include "cb2_rules.cuh"
#include "cb2_launch.cuh"

namespace cb2 {

// ---------------------------------------------------------------------------
// Strip pass: one CTA per strip task, K generations per launch
// ---------------------------------------------------------------------------

// The instantiated (K, V, L, rows per step) plans; for each (K, V) the first
// entry is the default levels-per-warp, for each (K, V, L) the first entry
// the default rows per step.
template <class R>
static const std::vector<strip_variant>& variants_for() {
    static const std::vector<strip_variant> v = {
        make_variant<R, 1, 2, 1>(),  make_variant<R, 1, 1, 1>(),  make_variant<R, 1, 4, 1>(),
        make_variant<R, 2, 2, 2>(),  make_variant<R, 2, 2, 1>(),  make_variant<R, 2, 1, 2>(),
        make_variant<R, 4, 2, 4>(),  make_variant<R, 4, 2, 2>(),  make_variant<R, 4, 1, 4>(),
        make_variant<R, 4, 4, 2>(),  make_variant<R, 8, 2, 4>(),  make_variant<R, 8, 2, 2>(),
        make_variant<R, 8, 1, 8>(),  make_variant<R, 8, 1, 4>(),  make_variant<R, 8, 4, 2>(),
        make_variant<R, 16, 2, 2>(), make_variant<R, 16, 2, 4>(), make_variant<R, 16, 4, 2>(),
        make_variant<R, 16, 1, 4>(), make_variant<R, 8, 2, 8>(),  make_variant<R, 16, 1, 16>(),
        make_variant<R, 4, 4, 4>(),
        make_variant<R, 16, 2, 8, 4>(), make_variant<R, 16, 2, 8, 2>(), make_variant<R, 16, 2, 4, 4>(),
        make_variant<R, 16, 2, 16, 4>(), make_variant<R, 16, 1, 16, 4>(),
        make_variant<R, 32, 2, 16, 4>(), make_variant<R, 32, 2, 8, 4>(), make_variant<R, 32, 2, 8, 2>(),
        make_variant<R, 32, 2, 4, 4>(), make_variant<R, 32, 1, 16, 4>(), make_variant<R, 32, 1, 32, 4>(),
        // short chains with two or four rows per step, so that rules which
        // evaluate rows in pairs (has_pairs) do so at every depth
        make_variant<R, 1, 2, 1, 2>(), make_variant<R, 1, 2, 1, 4>(), make_variant<R, 2, 2, 2, 2>(),
        make_variant<R, 2, 2, 2, 4>(), make_variant<R, 2, 2, 1, 4>(), make_variant<R, 4, 2, 4, 4>(),
        make_variant<R, 4, 2, 2, 4>(), make_variant<R, 8, 2, 8, 4>(), make_variant<R, 8, 2, 4, 4>(),
    };
    return v;
}

const std::vector<strip_variant>& strip_variants(int automaton) {
    static const std::vector<strip_variant> none;
    switch (automaton) {
    case 0: return variants_for<game_of_life>();
    case 1: return variants_for<wire>();
    case 2: return variants_for<excitable>();
    default: return automaton >= kNumBuiltin && automaton < automaton_count() ? generic_variants(automaton - kNumBuiltin)
                                                                               : none;
    }
}

const strip_variant* find_variant(int automaton, int k, int v, int l, int r) {
    for (const strip_variant& sv : strip_variants(automaton))
        if (sv.k == k && (v == 0 || sv.v == v) && (l == 0 || sv.l == l) && (r == 0 || sv.r == r)) return &sv;
    return nullptr;
}

void strip_counts(const grid_geom& g, int v, int tile_rows, int* nsx, int* nsy) {
    const int own = 32 * v - 2;
    *nsx = (g.wd + own - 1) / own;
    *nsy = (g.h + tile_rows - 1) / tile_rows;
}

static int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    return sms;
}

int resident_strip_tasks(const strip_variant& sv) {
    static std::mutex mu;
    static std::map<const void*, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(sv.fn);
    if (it != cache.end()) return it->second;
    cudaFuncSetAttribute(sv.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sv.smem_bytes);
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, sv.fn, sv.threads, sv.smem_bytes);
    const int n = std::max(1, blocks) * sm_count();
    cache[sv.fn] = n;
    return n;
}

int auto_tile_rows(const grid_geom& g, const strip_variant& sv) {
    const int resident = resident_strip_tasks(sv);
    int nsx, nsy;
    strip_counts(g, sv.v, 1, &nsx, &nsy);
    // One wave: as many row tasks per column as fit beside the other columns.
    const int per_column = std::max(1, resident / std::max(1, nsx));
    int rows = (g.h + per_column - 1) / per_column;
    // Keep the 2K halo rows of each task small against its own rows.
    rows = std::max(rows, 8 * sv.k);
    return std::min(rows, (int)g.h);
}

cudaError_t launch_strip_window(const grid_geom& g, const uint32_t* in, uint32_t* out, const run_plan& plan,
                                int y_base, int rows_out, cudaStream_t stream, int64_t t0, uint64_t seed,
                                int64_t y_global0, int64_t global_h) {
    const strip_variant* sv = find_variant(g.automaton, plan.k, plan.v, plan.l, plan.r);
    if (!sv || rows_out < 1 || y_base < 0 || y_base + rows_out > g.h) return cudaErrorInvalidValue;
    resident_strip_tasks(*sv);  // sets the kernel's shared-memory attribute once
    strip_launch a;
    a.in = in;
    a.out = out;
    a.plane_words = g.plane_words;
    a.wd = g.wd;
    a.h = g.h;
    a.tile_rows = plan.tile_rows;
    a.y_base = y_base;
    a.rows_out = rows_out;
    a.t0 = t0;
    a.seed = seed;
    a.y_global0 = y_global0;
    a.global_h = global_h > 0 ? global_h : g.h;
    grid_geom window = g;
    window.h = rows_out;
    strip_counts(window, plan.v, plan.tile_rows, &a.nsx, &a.nsy);
    const int64_t tasks = (int64_t)a.nsx * a.nsy;
    void* args[] = {&a};
    return cudaLaunchKernel(sv->fn, dim3((unsigned)tasks), dim3(sv->threads), args, (size_t)sv->smem_bytes, stream);
}

cudaError_t launch_strip_pass(const grid_geom& g, const uint32_t* in, uint32_t* out, const run_plan& plan,
                              cudaStream_t stream, int64_t t0, uint64_t seed) {
    return launch_strip_window(g, in, out, plan, 0, g.h, stream, t0, seed);
}

// ---------------------------------------------------------------------------
// Seeded input generator: cell i = y*X + x draws u = mix(seed + (i+1)*gamma)
// >> 11 (SplitMix64, 53 uniform bits); its state index is the number of
// cumulative thresholds <= u.
// ---------------------------------------------------------------------------

struct thr_pack {
    unsigned long long t[kMaxThresholds];
    int n;
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Row y of the planes holds global row (row0 + y) mod global_rows.
__global__ void fill_random_kernel(uint32_t* planes, int64_t plane_words, int32_t wd, int64_t x_size, int P,
                                   uint64_t seed, thr_pack thr, int64_t row0, int64_t global_rows) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < plane_words; w += stride) {
        const int64_t y = w / wd, xw = w - y * wd;
        int64_t gy = (row0 + y) % global_rows;
        if (gy < 0) gy += global_rows;
        const uint64_t i0 = (uint64_t)(gy * x_size + xw * 32);
        uint32_t out[kMaxPlanes] = {};
#pragma unroll 4
        for (int j = 0; j < 32; ++j) {
            const uint64_t u = mix64(seed + (i0 + j + 1) * 0x9E3779B97F4A7C15ull) >> 11;
            uint32_t s = 0;
            for (int t = 0; t < thr.n; ++t) s += u >= thr.t[t];
#pragma unroll
            for (int p = 0; p < kMaxPlanes; ++p) out[p] |= ((s >> p) & 1u) << j;
        }
        for (int p = 0; p < P; ++p) planes[p * plane_words + w] = out[p];
    }
}

static unsigned grid_for(int64_t items, int threads) {
    const int64_t b = (items + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 64));
}

cudaError_t launch_fill_random_rows(const grid_geom& g, uint32_t* planes, uint64_t seed, const uint64_t* thr, int nthr,
                                    int64_t row0, int64_t global_rows, cudaStream_t s) {
    if (nthr < 0 || nthr > kMaxThresholds || global_rows < 1) return cudaErrorInvalidValue;
    thr_pack tp{};
    for (int i = 0; i < nthr; ++i) tp.t[i] = thr[i];
    tp.n = nthr;
    fill_random_kernel<<<grid_for(g.plane_words, 256), 256, 0, s>>>(planes, g.plane_words, g.wd, g.x_size, g.planes,
                                                                     seed, tp, row0, global_rows);
    return cudaGetLastError();
}

cudaError_t launch_fill_random(const grid_geom& g, uint32_t* planes, uint64_t seed, const uint64_t* thr, int nthr,
                               cudaStream_t s) {
    return launch_fill_random_rows(g, planes, seed, thr, nthr, 0, g.h, s);
}

// ---------------------------------------------------------------------------
// Standard layout (one state index per cell, 1 or 4 bytes) <-> planes.
// Thread per 32-cell plane word; rows are whole words (x_size % 32 == 0).
// ---------------------------------------------------------------------------

template <typename cell_t>
__global__ void pack_cells_kernel(const cell_t* __restrict__ cells, int64_t plane_words, int32_t wd, int64_t x_size,
                                  int P, int states, uint32_t* __restrict__ planes, unsigned* bad) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const uint32_t max_state = (uint32_t)states - 1u;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < plane_words; w += stride) {
        const int64_t y = w / wd, xw = w - y * wd;
        const cell_t* src = cells + y * x_size + xw * 32;
        uint32_t out[kMaxPlanes] = {};
        bool any_bad = false;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const uint32_t s = (uint32_t)src[j];
            any_bad |= s > max_state;
#pragma unroll
            for (int p = 0; p < kMaxPlanes; ++p) out[p] |= ((s >> p) & 1u) << j;
        }
        if (any_bad) atomicOr(bad, 1u);
        for (int p = 0; p < P; ++p) planes[p * plane_words + w] = out[p];
    }
}

template <typename cell_t>
__global__ void unpack_cells_kernel(const uint32_t* __restrict__ planes, int64_t plane_words, int32_t wd,
                                    int64_t x_size, int P, cell_t* __restrict__ cells) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < plane_words; w += stride) {
        const int64_t y = w / wd, xw = w - y * wd;
        uint32_t in[kMaxPlanes] = {};
        for (int p = 0; p < P; ++p) in[p] = planes[p * plane_words + w];
        cell_t* dst = cells + y * x_size + xw * 32;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            uint32_t s = 0;
#pragma unroll
            for (int p = 0; p < kMaxPlanes; ++p) s |= ((in[p] >> j) & 1u) << p;
            dst[j] = (cell_t)s;
        }
    }
}

cudaError_t launch_pack_cells(const grid_geom& g, const void* cells, int cell_bytes, uint32_t* planes,
                              unsigned* bad_flag, cudaStream_t s) {
    const unsigned blocks = grid_for(g.plane_words, 256);
    if (cell_bytes == 1)
        pack_cells_kernel<uint8_t><<<blocks, 256, 0, s>>>((const uint8_t*)cells, g.plane_words, g.wd, g.x_size,
                                                           g.planes, g.states, planes, bad_flag);
    else if (cell_bytes == 4)
        pack_cells_kernel<uint32_t><<<blocks, 256, 0, s>>>((const uint32_t*)cells, g.plane_words, g.wd, g.x_size,
                                                            g.planes, g.states, planes, bad_flag);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_unpack_cells(const grid_geom& g, const uint32_t* planes, void* cells, int cell_bytes,
                                cudaStream_t s) {
    const unsigned blocks = grid_for(g.plane_words, 256);
    if (cell_bytes == 1)
        unpack_cells_kernel<uint8_t><<<blocks, 256, 0, s>>>(planes, g.plane_words, g.wd, g.x_size, g.planes,
                                                             (uint8_t*)cells);
    else if (cell_bytes == 4)
        unpack_cells_kernel<uint32_t><<<blocks, 256, 0, s>>>(planes, g.plane_words, g.wd, g.x_size, g.planes,
                                                              (uint32_t*)cells);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// bit_array layout (memory/bit_array_grid.hpp:80-333): cells_per_word =
// W / P whole states per W-bit word, cell i = y*X + x at word i / cpw, bit
// (i % cpw) * P.  A word never spans two rows (X % cpw == 0).
// ---------------------------------------------------------------------------

template <typename word_t>
__global__ void bit_array_to_planes_kernel(const word_t* __restrict__ words, int64_t plane_words, int32_t wd,
                                           int64_t x_size, int P, uint32_t* __restrict__ planes) {
    constexpr int W = sizeof(word_t) * 8;
    const int cpw = W / P;
    const word_t mask = (word_t)((1u << P) - 1u);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < plane_words; w += stride) {
        const int64_t y = w / wd, xw = w - y * wd;
        const int64_t i0 = y * x_size + xw * 32;
        int64_t wi = i0 / cpw;
        int r = (int)(i0 - wi * cpw);
        word_t cur = words[wi];
        uint32_t out[kMaxPlanes] = {};
        for (int j = 0; j < 32; ++j) {
            const uint32_t s = (uint32_t)((cur >> (r * P)) & mask);
#pragma unroll
            for (int p = 0; p < kMaxPlanes; ++p) out[p] |= ((s >> p) & 1u) << j;
            if (++r == cpw && j < 31) {
                r = 0;
                cur = words[++wi];
            }
        }
        for (int p = 0; p < P; ++p) planes[p * plane_words + w] = out[p];
    }
}

template <typename word_t>
__global__ void planes_to_bit_array_kernel(const uint32_t* __restrict__ planes, int64_t plane_words, int32_t wd,
                                           int64_t x_size, int64_t n_words, int P, word_t* __restrict__ words) {
    constexpr int W = sizeof(word_t) * 8;
    const int cpw = W / P;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t wi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; wi < n_words; wi += stride) {
        const int64_t i0 = wi * cpw;
        const int64_t y = i0 / x_size, x0 = i0 - y * x_size;
        word_t out = 0;
        int64_t pw = -1;
        uint32_t in[kMaxPlanes] = {};
        for (int j = 0; j < cpw; ++j) {
            const int64_t x = x0 + j;
            if ((x >> 5) != pw) {
                pw = x >> 5;
                for (int p = 0; p < P; ++p) in[p] = planes[p * plane_words + y * wd + pw];
            }
            word_t s = 0;
            for (int p = 0; p < P; ++p) s |= (word_t)((in[p] >> (x & 31)) & 1u) << p;
            out |= s << (j * P);
        }
        words[wi] = out;
    }
}

cudaError_t launch_bit_array_to_planes(const grid_geom& g, const void* words, int word_bits, uint32_t* planes,
                                       cudaStream_t s) {
    const unsigned blocks = grid_for(g.plane_words, 256);
    if (word_bits == 32)
        bit_array_to_planes_kernel<uint32_t><<<blocks, 256, 0, s>>>((const uint32_t*)words, g.plane_words, g.wd,
                                                                     g.x_size, g.planes, planes);
    else if (word_bits == 64)
        bit_array_to_planes_kernel<unsigned long long><<<blocks, 256, 0, s>>>(
            (const unsigned long long*)words, g.plane_words, g.wd, g.x_size, g.planes, planes);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_planes_to_bit_array(const grid_geom& g, const uint32_t* planes, void* words, int word_bits,
                                       cudaStream_t s) {
    const int cpw = word_bits / g.planes;
    const int64_t n_words = g.x_size * g.y_size / cpw;
    const unsigned blocks = grid_for(n_words, 256);
    if (word_bits == 32)
        planes_to_bit_array_kernel<uint32_t><<<blocks, 256, 0, s>>>(planes, g.plane_words, g.wd, g.x_size, n_words,
                                                                     g.planes, (uint32_t*)words);
    else if (word_bits == 64)
        planes_to_bit_array_kernel<unsigned long long><<<blocks, 256, 0, s>>>(
            planes, g.plane_words, g.wd, g.x_size, n_words, g.planes, (unsigned long long*)words);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// tiled_bit_planes layout (memory/tiled_bit_planes_grid.hpp:244-287): a W-bit
// word is an 8 x (W/8) tile, bit (x%8) + 8*(y%th).  Byte r of tile word
// (xt, yt) is therefore byte xt of linear row yt*th + r: a byte gather.
// ---------------------------------------------------------------------------

__global__ void tiled_to_planes_kernel(const uint8_t* __restrict__ tiled, int64_t plane_words, int32_t wd,
                                       int64_t x_size, int th, int P, uint32_t* __restrict__ planes) {
    const int64_t xt_n = x_size / 8;
    const int64_t plane_bytes = plane_words * 4;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < plane_words; w += stride) {
        const int64_t y = w / wd, xw = w - y * wd;
        const int64_t base = ((y / th) * xt_n + xw * 4) * th + (y % th);
        for (int p = 0; p < P; ++p) {
            const uint8_t* src = tiled + p * plane_bytes + base;
            planes[p * plane_words + w] = (uint32_t)src[0] | ((uint32_t)src[th] << 8) |
                                          ((uint32_t)src[2 * th] << 16) | ((uint32_t)src[3 * th] << 24);
        }
    }
}

__global__ void planes_to_tiled_kernel(const uint32_t* __restrict__ planes, int64_t plane_words, int32_t wd,
                                       int64_t x_size, int th, int P, uint8_t* __restrict__ tiled) {
    const int64_t xt_n = x_size / 8;
    const int64_t plane_bytes = plane_words * 4;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < plane_words; w += stride) {
        const int64_t y = w / wd, xw = w - y * wd;
        const int64_t base = ((y / th) * xt_n + xw * 4) * th + (y % th);
        for (int p = 0; p < P; ++p) {
            const uint32_t v = planes[p * plane_words + w];
            uint8_t* dst = tiled + p * plane_bytes + base;
            dst[0] = (uint8_t)v;
            dst[th] = (uint8_t)(v >> 8);
            dst[2 * th] = (uint8_t)(v >> 16);
            dst[3 * th] = (uint8_t)(v >> 24);
        }
    }
}

cudaError_t launch_tiled_to_planes(const grid_geom& g, const void* tiled, int word_bits, uint32_t* planes,
                                   cudaStream_t s) {
    if (word_bits != 32 && word_bits != 64) return cudaErrorInvalidValue;
    tiled_to_planes_kernel<<<grid_for(g.plane_words, 256), 256, 0, s>>>(
        (const uint8_t*)tiled, g.plane_words, g.wd, g.x_size, word_bits / 8, g.planes, planes);
    return cudaGetLastError();
}

cudaError_t launch_planes_to_tiled(const grid_geom& g, const uint32_t* planes, void* tiled, int word_bits,
                                   cudaStream_t s) {
    if (word_bits != 32 && word_bits != 64) return cudaErrorInvalidValue;
    planes_to_tiled_kernel<<<grid_for(g.plane_words, 256), 256, 0, s>>>(planes, g.plane_words, g.wd, g.x_size,
                                                                        word_bits / 8, g.planes, (uint8_t*)tiled);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Checksum (memory/standard_grid.hpp:182-218): 4 x 4 tiles of ceil(X/4) x
// ceil(Y/4) cells, sum of state VALUES per tile.  Counted from the planes
// with popcounts of per-state minterms under per-tile column masks.
// ---------------------------------------------------------------------------

struct value_pack {
    long long v[1 << kMaxPlanes];
};

// Sums rows [row_first, row_first + row_count) of the planes, which are
// global rows global_row0 + (y - row_first) of a grid global_rows tall.
__global__ void checksum_kernel(const uint32_t* __restrict__ planes, int64_t plane_words, int32_t wd,
                                int64_t x_size, int64_t row_first, int64_t row_count, int64_t global_row0,
                                int64_t global_rows, int P, value_pack vals, unsigned long long* sums) {
    __shared__ unsigned long long acc[16];
    if (threadIdx.x < 16) acc[threadIdx.x] = 0;
    __syncthreads();
    const int64_t tw = (x_size + 3) / 4, th = (global_rows + 3) / 4;
    const int nstates = 1 << P;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t words = row_count * wd;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < words; k += stride) {
        const int64_t yr = k / wd, xw = k - yr * wd;
        const int64_t w = (row_first + yr) * wd + xw;
        const int ty = (int)((global_row0 + yr) / th);
        uint32_t in[kMaxPlanes] = {};
        for (int p = 0; p < P; ++p) in[p] = planes[p * plane_words + w];
        const int64_t x0 = xw * 32, x1 = x0 + 32;
        for (int64_t tx = x0 / tw; tx < 4 && tx * tw < x1; ++tx) {
            const int64_t lo = x0 > tx * tw ? x0 : tx * tw, hi = x1 < (tx + 1) * tw ? x1 : (tx + 1) * tw;
            const int nbits = (int)(hi - lo), shift = (int)(lo - x0);
            const uint32_t m = (nbits >= 32 ? 0xffffffffu : ((1u << nbits) - 1u)) << shift;
            long long sum = 0;
            for (int s = 0; s < nstates; ++s) {
                uint32_t mt = m;
                for (int p = 0; p < P; ++p) mt &= ((s >> p) & 1) ? in[p] : ~in[p];
                sum += vals.v[s] * (long long)__popc(mt);
            }
            if (sum) atomicAdd(&acc[ty * 4 + tx], (unsigned long long)sum);
        }
    }
    __syncthreads();
    if (threadIdx.x < 16 && acc[threadIdx.x]) atomicAdd(&sums[threadIdx.x], acc[threadIdx.x]);
}

cudaError_t launch_checksum_rows(const grid_geom& g, const uint32_t* planes, const int64_t* values, int nvalues,
                                 int64_t row_first, int64_t row_count, int64_t global_row0, int64_t global_rows,
                                 unsigned long long* sums, cudaStream_t s) {
    if (row_first < 0 || row_count < 0 || row_first + row_count > g.h || global_row0 < 0 ||
        global_row0 + row_count > global_rows)
        return cudaErrorInvalidValue;
    value_pack vp{};
    for (int i = 0; i < (1 << kMaxPlanes); ++i) vp.v[i] = i < nvalues ? values[i] : i;
    checksum_kernel<<<grid_for(row_count * g.wd, 256), 256, 0, s>>>(planes, g.plane_words, g.wd, g.x_size, row_first,
                                                                    row_count, global_row0, global_rows, g.planes, vp,
                                                                    sums);
    return cudaGetLastError();
}

cudaError_t launch_checksum(const grid_geom& g, const uint32_t* planes, const int64_t* values, int nvalues,
                            unsigned long long* sums, cudaStream_t s) {
    return launch_checksum_rows(g, planes, values, nvalues, 0, g.h, 0, g.h, sums, s);
}

// ---------------------------------------------------------------------------
// Integer-pipe probe: eight independent chains of three-input logic ops per
// lane (the same LOP3 class the rule networks compile to).
// ---------------------------------------------------------------------------

__global__ void lop3_probe_kernel(uint32_t* sink, int iters) {
    uint32_t r[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) r[i] = threadIdx.x * 0x9E3779B9u + i * 0x85EBCA6Bu + blockIdx.x;
    const uint32_t a = 0x12345678u ^ blockIdx.x, b = 0x9abcdef0u ^ threadIdx.x;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
#pragma unroll
            for (int i = 0; i < 8; ++i)
                asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(r[i]) : "r"(a), "r"(b ^ (uint32_t)u));
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) x ^= r[i];
    if (x == 0x7fffffffu) sink[0] = x;  // keeps the chains alive
}

cudaError_t launch_lop3_probe(uint32_t* sink, int blocks, int threads, int iters, cudaStream_t s) {
    lop3_probe_kernel<<<blocks, threads, 0, s>>>(sink, iters);
    return cudaGetLastError();
}

} // namespace cb2
