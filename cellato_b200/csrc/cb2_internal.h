// cb2_internal.h -- declarations shared by the library's translation units.
// Not part of the public C-ABI (include/cellato_b200.h is).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace cb2 {

constexpr int kMaxPlanes = 5;       // bit-planes of the largest dictionary (32 states)
constexpr int kNumBuiltin = 3;      // automata with hand-written networks: ids 0, 1, 2
constexpr int kMaxThresholds = 31;  // up to 32 states
constexpr int kRingDepth = 8;       // input rows kept in flight per strip task
constexpr uint64_t kDefaultSeed = 42;  // run_params::seed

// Geometry of one device grid: P planes of h rows x wd 32-bit words.
struct grid_geom {
    int automaton;
    int planes;
    int states;              // dictionary size: indexes >= states are not states
    int64_t x_size, y_size;  // cells
    int32_t wd, h;           // 32-bit words per row, rows
    int64_t plane_words;     // wd * h
};

// Tuning knobs for one single-grid run.
struct run_plan {
    int k;          // generations per launch (1, 2, 4, 8, 16 or 32)
    int v;          // 32-bit words per lane (1, 2 or 4)
    int l;          // levels (generations) per warp; the CTA has k / l warps
    int r;          // rows each warp takes per barrier (1, 2 or 4)
    int tile_rows;  // output rows per strip task
};

// One instantiated strip kernel.
struct strip_variant {
    int k, v, l, r;
    const void* fn;
    int threads;
    int smem_bytes;
};

// The automaton registry: ids 0..2 are the hand-written networks, ids from
// 3 the DSL automata lowered by cb2_ast.cuh (cb2_generic.cu; absent when the
// library was built without the Cellato headers).
struct automaton_desc {
    const char* name;
    int planes;
    int states;
    const int64_t* values;  // dictionary index -> state value (the checksum sums values)
    uint64_t fingerprint = 0;  // of the Cellato config's rule and dictionary (0: unknown)
};
int automaton_count();
const automaton_desc* automaton_at(int id);  // nullptr for an unknown id
int planes_of(int automaton);
const char* name_of(int automaton);
int find_automaton(const char* name);
// Lowered DSL automata (cb2_generic.cu): how many, and their descriptors and
// kernels, indexed from 0 (= automaton id kNumBuiltin).
int generic_count();
const automaton_desc* generic_desc(int i);
// Fingerprint (include/cellato_b200/fingerprint.hpp) of the Cellato config a
// hand-written network (id < kNumBuiltin) computes, 0 when the library was
// built without the Cellato headers.
uint64_t builtin_fingerprint(int id);

// Launches one K-generation strip pass over a whole grid (in -> out); the
// input is generation t0 (read by time-dependent rules), seed the run's
// random seed (read by stochastic rules).
cudaError_t launch_strip_pass(const grid_geom& g, const uint32_t* in, uint32_t* out, const run_plan& plan,
                              cudaStream_t stream, int64_t t0 = 0, uint64_t seed = kDefaultSeed);
// The same for output rows [y_base, y_base + rows_out) only (input rows wrap mod g.h).
// y_global0 / global_h place the planes' rows in a larger grid (a band of
// it): rules that read the row see global rows (0 = the planes are the grid).
cudaError_t launch_strip_window(const grid_geom& g, const uint32_t* in, uint32_t* out, const run_plan& plan,
                                int y_base, int rows_out, cudaStream_t stream, int64_t t0 = 0,
                                uint64_t seed = kDefaultSeed, int64_t y_global0 = 0, int64_t global_h = 0);
// Strip tasks per column and per row for a plan.
void strip_counts(const grid_geom& g, int v, int tile_rows, int* nsx, int* nsy);
// The instantiated kernels of an automaton, and the first one matching a
// plan (v, l or r of 0 match anything).
const std::vector<strip_variant>& strip_variants(int automaton);
const std::vector<strip_variant>& generic_variants(int i);  // of lowered automaton i
const strip_variant* find_variant(int automaton, int k, int v, int l, int r = 0);
// Output rows per task so that one launch fills the GPU about once.
int auto_tile_rows(const grid_geom& g, const strip_variant& sv);
// Number of strip-task CTAs resident at once on this device.
int resident_strip_tasks(const strip_variant& sv);

// Layout conversions between host images and device planes (device -> device).
cudaError_t launch_pack_cells(const grid_geom& g, const void* cells, int cell_bytes, uint32_t* planes,
                              unsigned* bad_flag, cudaStream_t s);
cudaError_t launch_unpack_cells(const grid_geom& g, const uint32_t* planes, void* cells, int cell_bytes,
                                cudaStream_t s);
cudaError_t launch_bit_array_to_planes(const grid_geom& g, const void* words, int word_bits, uint32_t* planes,
                                       cudaStream_t s);
cudaError_t launch_planes_to_bit_array(const grid_geom& g, const uint32_t* planes, void* words, int word_bits,
                                       cudaStream_t s);
cudaError_t launch_tiled_to_planes(const grid_geom& g, const void* tiled, int word_bits, uint32_t* planes,
                                   cudaStream_t s);
cudaError_t launch_planes_to_tiled(const grid_geom& g, const uint32_t* planes, void* tiled, int word_bits,
                                   cudaStream_t s);
cudaError_t launch_fill_random(const grid_geom& g, uint32_t* planes, uint64_t seed, const uint64_t* thr, int nthr,
                               cudaStream_t s);
// Row y of the planes gets global row (row0 + y) mod global_rows of the seeded grid.
cudaError_t launch_fill_random_rows(const grid_geom& g, uint32_t* planes, uint64_t seed, const uint64_t* thr, int nthr,
                                    int64_t row0, int64_t global_rows, cudaStream_t s);
// Adds the 16 tile sums of state values into sums[16] (which the caller zeroes).
cudaError_t launch_checksum(const grid_geom& g, const uint32_t* planes, const int64_t* values, int nvalues,
                            unsigned long long* sums, cudaStream_t s);
// The same for rows [row_first, row_first + row_count), which are global rows
// global_row0.. of a grid global_rows tall (a band's share of the global tiles).
cudaError_t launch_checksum_rows(const grid_geom& g, const uint32_t* planes, const int64_t* values, int nvalues,
                                 int64_t row_first, int64_t row_count, int64_t global_row0, int64_t global_rows,
                                 unsigned long long* sums, cudaStream_t s);

// Integer-pipe peak probe: `iters` rounds of independent 3-input logic ops.
cudaError_t launch_lop3_probe(uint32_t* sink, int blocks, int threads, int iters, cudaStream_t s);
// Logic ops one lane of the probe kernel issues per iteration.
constexpr int kLop3ProbeOpsPerIter = 64;

// Thread-local error message for cb2_last_error().
void set_error(const std::string& msg);

}  // namespace cb2

struct cb2_tuning;

namespace cb2 {

// Validates a grid size for an automaton and fills its geometry.
int make_geom(int automaton, int64_t x, int64_t y, grid_geom* g);
// The run plan for a grid: the fields of `t` that are 0 are chosen from the
// tuning table or the defaults.
int resolve_plan(const grid_geom& g, const cb2_tuning* t, run_plan* plan);
// Launches `steps` generations starting in bufs[cur], alternating between the
// two buffers; *result is the index of the buffer holding the result.
int run_chunks(const grid_geom& g, uint32_t* const bufs[2], int cur, int64_t steps, const cb2_tuning* tuning,
               cudaStream_t stream, int* result, int64_t t0 = 0, uint64_t seed = kDefaultSeed);

} // namespace cb2

// An owning device grid (the opaque cb2_grid of the C-ABI).
struct cb2_grid {
    cb2::grid_geom g{};
    uint32_t* buf[2] = {nullptr, nullptr};  // the double buffer; buf[cur] holds the current generation
    int cur = 0;
    int64_t time_step = 0;
    uint64_t seed = cb2::kDefaultSeed;  // random seed of stochastic rules
    void* staging = nullptr;  // device copy of a host image for layout conversion
    size_t staging_bytes = 0;
    unsigned* flag = nullptr;  // device error flag of the conversion kernels
    unsigned long long* sums = nullptr;
    int device = 0;
};
