// cb2_batch.h -- the batch engine shared by cb2_batch_* and the serving loop
// (internal; the C-ABI is include/cellato_b200.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cb2_internal.h"

namespace cb2 {

// One CTA's work: one strip (groups == 0), `groups` exact-wrap copies of a
// narrow grid's row (groups > 0), or -groups row bands of a narrow last
// strip side by side in the warp (groups < 0, band_geom), for one chunk of k
// generations.  The tasks of a chunk tile the grid as nsy rows of nsx tasks;
// (tx, ty) is this one.
struct batch_task {
    int32_t grid;      // index into the grid table
    int32_t chunk;     // reads buffer chunk & 1, writes the other one
    int32_t dep_base;  // index of the previous chunk's first task, -1 for chunk 0
    int32_t rows;      // output rows of the task (strip), or of each group / band
    int16_t k;         // generations (1 .. 32)
    int16_t groups;    // 0 = strip task, > 0 exact-wrap groups, < 0 row bands
    int16_t nsx, nsy;  // tasks per tile row / tile rows of this grid's chunks
    int16_t tx, ty;    // this task's tile
    int32_t y0;        // first output row; the last tile row absorbs the remainder,
                       // so no tile is shorter than K and a task's halo stays
                       // within its neighbouring tiles
};
static_assert(sizeof(batch_task) == 32, "batch_task is one 32-byte sector");

struct batch_grid_desc {
    uint32_t* buf[2];  // buf[0] holds the current generation when a run starts
    int64_t plane_words;
    int64_t t0;     // generation of the grid when the run starts (advanced on the device after each run)
    uint64_t seed;  // random seed of stochastic rules
    int64_t steps;  // generations of a run
    int32_t wd, h;
    int32_t automaton;
    int32_t kmain;  // K of the full chunks; nfull of them, then the remainder rem < kmain
    int32_t nfull, rem;
};

struct batch_args {
    const batch_task* tasks;
    const unsigned* ntasks;  // in device memory, so one captured graph runs any list
    const batch_grid_desc* grids;
    unsigned* task_done;  // per task: 1 once its outputs are written
    unsigned* head;       // next task to take
    unsigned* error;      // 0, or 1 + the task whose wait ran out
    long long spin_limit;
};

struct batch_item {
    cb2_grid* grid;
    int64_t steps;
    int cur;        // the grid's current buffer when the schedule was built
    int64_t t0;     // the grid's generation when the schedule was built
    uint64_t seed;  // and its random seed
};

struct batch_tiling {
    int temporal_steps = 8;  // K of full chunks
    int tile_rows = 256;     // output rows per strip task of a hand-written network
    // ... of a lowered DSL rule.  Its tasks do ~100x the work per row, so with long
    // tiles a long-running grid's chain of chunks, not the total work, sets the
    // run's length (1024 mixed DSL grids: 1.87 Tcell/s at 256 rows, 2.19 at 128,
    // 2.31 at 64, 2.02 at 32; the networks' mix is best at 256).
    int lowered_tile_rows = 64;
    int rows_for(int automaton) const { return automaton >= kNumBuiltin ? lowered_tile_rows : tile_rows; }
};

// The two kernels of a batch: the hand-written networks alone, or every
// registered automaton (the lowered DSL rules need more registers and shared
// memory, so they get a kernel of their own).
enum batch_kind { kBatchBuiltin = 0, kBatchAll = 1 };

// Warps of a CTA (one task) in each kind's kernel.  Two warps per task for
// the networks (four levels each, twice the resident CTAs) measured slower:
// 18.1 against 19.1 Tcell/s on the batched workload, 12.4 against 15.0 served
// at 20000 req/s -- the longer chain links cost more than the occupancy gains.
constexpr int kBatchKindWarps[2] = {4, 4};

// The kernel of kind kBatchAll (cb2_generic_batch.cu); null when the library
// has no lowered DSL automata.
const void* generic_batch_kernel();

// Device task list, counters and the captured launch graphs.
struct batch_engine {
    int device = 0;
    int kmax = 8;
    long long spin_limit = 0;
    int task_cap = 0, grid_cap = 0;
    int ntasks = 0, ngrids = 0;
    int kind = kBatchBuiltin;  // the kernel the built schedule needs
    double cells_per_run = 0;
    int blocks = 0;           // persistent CTAs of the kernel of `kind`
    int kind_blocks[2] = {0, 0};
    batch_task* d_tasks = nullptr;
    batch_grid_desc* d_grids = nullptr;
    unsigned char* d_odd = nullptr;
    unsigned* d_counters = nullptr;  // head, error, ngrids (for the flip kernel), ntasks
    unsigned* d_task_done = nullptr; // per task
    batch_task* h_tasks = nullptr;   // pinned
    batch_grid_desc* h_grids = nullptr;
    unsigned char* h_odd = nullptr;
    unsigned* h_misc = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph[2] = {nullptr, nullptr};  // per kind
    cudaGraphExec_t exec[2] = {nullptr, nullptr};

    int init(int task_capacity, int grid_capacity, int kmax, long long spin_limit);
    void release();
    // Fills h_tasks / h_grids / h_odd with the schedule of `items`.
    int build(const std::vector<batch_item>& items, const batch_tiling& tiling);
    // Copies the schedule to the device (asynchronous on s).
    int upload(cudaStream_t s);
    // Replays the captured graph of the schedule's kind (captures it on first
    // use) on s.
    int launch(cudaStream_t s);
    // Waits for s and reports a timed-out wait as CB2_ETIMEOUT.
    int check(cudaStream_t s);
    // Queues a copy of the run's error word to pinned memory on s; after the
    // stream passed it, error_seen() reports it without synchronising.
    int read_error_async(cudaStream_t s);
    int error_seen();
    // Captures the launch graph of a kind now (launch does it on first use
    // otherwise).  kBatchAll fails when there are no lowered DSL automata.
    int capture(int kind = kBatchBuiltin);
};

} // namespace cb2
