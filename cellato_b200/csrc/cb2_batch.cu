// cb2_batch.cu -- many independent grids in one persistent kernel.
//
// A batch advances each of its grids by that grid's own number of
// generations.  The work is cut into tasks: one task = one CTA running the
// level pipeline (pipe_run_rows, cb2_pipe.cuh) over one strip of one grid
// for one chunk of K generations, its K levels split over the CTA's four
// warps, four rows per barrier.  Splitting the levels divides a task's
// latency, and with it the length of a grid's chain of chunks, by four (a
// task per warp: 15.9-18.0 Tcell/s; per CTA: 19.1 on the bench workload).
// Grids at most 16 words wide run in group geometry: the lanes hold several
// exact-wrap copies of the row, each over its own rows, so narrow grids do
// not waste the warp on halo.
//
// The tasks sit in a device array in schedule order.  A persistent kernel
// (one CTA per resident slot, one task at a time) takes tasks in that
// order from an atomic head index.  Chunk c of a grid reads buffer c&1 and
// writes the other.  The tasks of every chunk of a grid tile it the same
// way, and a task reads its own tile plus K rows and one word around it, so
// a task of chunk c waits only for the (up to) nine tasks of chunk c-1 on
// its own and the neighbouring tiles (torus wrap): they wrote everything it
// reads, and they are the only readers of the region it overwrites.  Chunks
// of one grid thus run as a wavefront instead of pass by pass.  Each task
// publishes a done flag (release); waiters acquire it.  A task only ever
// waits for tasks earlier in the order, which were taken by warps that are
// running, so the earliest unfinished task can always proceed.  The wait is still bounded (spin_limit): when it runs out,
// the warp records the task in an error word and every warp stops taking
// tasks, so a broken schedule ends the kernel with an error status instead
// of a hang.
//
// Order: by progress through the grid, (level + 1/2) / levels, so every
// grid's chain of levels is spread over the whole run and the longest
// chains do not run alone at the end; ties go to the grids with the most
// chunks.  A grid's levels keep their order, so every task still waits only
// for earlier tasks.  (Level-major order -- all grids' level c before any
// level c+1 -- left a tail of a few long-running grids: 15.9 against 18.1
// Tcell/s on 4096 mixed grids.)
//
// The launch (counter resets + kernel) is captured once in a CUDA graph and
// replayed; the task count lives in device memory, so the same graph runs
// any task list up to the engine's capacity (the serving loop relies on it).
//
// Two kernels share this schedule (cb2_batch_kernel.cuh): one over the
// hand-written networks alone, here, and one over every registered
// automaton, cb2_generic_batch.cu, which a batch holding a lowered DSL
// automaton runs.  There a task also takes its chunk's first generation
// (from the grid's run start and its chunk split) and the grid's seed, which
// stochastic and time-dependent rules read; the run start advances on the
// device after each run, so replays continue the grids' time.
// The batch kernels keep plain copies of the planes a rule passes on (cb2_rules.cuh fresh).
#define CB2_PLAIN_COPIES
#include "cellato_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "cb2_batch.h"
#include "cb2_batch_kernel.cuh"
#include "cb2_internal.h"
#include "cb2_rules.cuh"

namespace cb2 {

constexpr int kBuiltinPlanes = 3;  // the hand-written networks' largest P
constexpr int kBatchDefaultK = 32;      // cb2_batch_create's chunk length (capped at kBatchKMax with lowered rules)
constexpr int kBatchDefaultRows = 768;  // and its tile height for the hand-written networks
constexpr int kBuiltinRows = 4;    // rows each warp passes on per barrier (2: 18.3, 4: 19.1, 8: 16.6 Tcell/s)

// The hand-written networks: the kernel of kind kBatchBuiltin, one per
// longest chunk KMAX (4, 8, 16 or 32 generations), so that a batch of short
// chunks does not carry the registers of the longer pipelines.
template <int KMAX>
struct builtin_rules {
    static constexpr int kWarps = kBatchKindWarps[kBatchBuiltin];
    static constexpr int kSmemWords = batch_smem_words(kBuiltinPlanes, kBuiltinRows, kWarps);
    static constexpr bool kTimed = false;  // the networks read neither time, seed nor global rows
    __device__ __forceinline__ static void run(int automaton, int k, const strip_task& t, const lane_geom<1>& geom,
                                               uint32_t* smem) {
        switch (automaton) {
        case 0: batch_run_rule<game_of_life, KMAX, kBuiltinRows, kSmemWords, kWarps>(t, k, geom, smem); break;
        case 1: batch_run_rule<wire, KMAX, kBuiltinRows, kSmemWords, kWarps>(t, k, geom, smem); break;
        default: batch_run_rule<excitable, KMAX, kBuiltinRows, kSmemWords, kWarps>(t, k, geom, smem); break;
        }
    }
};

// After a run, a grid that took an odd number of chunks holds its result in
// buffer 1: swap so that buffer 0 is again the current generation.  Every
// grid's generation advances by its steps, so a replay of the same schedule
// continues the grids' time.
__global__ void batch_flip_kernel(batch_grid_desc* grids, const unsigned char* odd, const unsigned* n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (int)*n) {
        if (odd[i]) {
            uint32_t* t = grids[i].buf[0];
            grids[i].buf[0] = grids[i].buf[1];
            grids[i].buf[1] = t;
        }
        grids[i].t0 += grids[i].steps;
    }
}

static const void* batch_kernel_for(int kind, int kmax) {
    if (kind == kBatchAll) return generic_batch_kernel();
    if (kmax >= 32) return (const void*)batch_kernel<builtin_rules<32>>;
    if (kmax >= 16) return (const void*)batch_kernel<builtin_rules<16>>;
    return kmax >= 8 ? (const void*)batch_kernel<builtin_rules<8>> : (const void*)batch_kernel<builtin_rules<4>>;
}

// ---- engine -------------------------------------------------------------------------------------

static int efail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

static int ecuda(cudaError_t e, const char* what) {
    cudaGetLastError();
    return efail(e == cudaErrorMemoryAllocation ? CB2_ENOMEM : CB2_ECUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

int batch_engine::init(int task_capacity, int grid_capacity, int kmax_, long long spin_limit_) {
    kmax = kmax_ >= 32 ? 32 : kmax_ >= 16 ? 16 : (kmax_ >= 8 ? 8 : 4);
    spin_limit = spin_limit_ > 0 ? spin_limit_ : (1ll << 23);
    task_cap = std::max(1, task_capacity);
    grid_cap = std::max(1, grid_capacity);
    cudaGetDevice(&device);
    cudaError_t e = cudaMalloc(&d_tasks, sizeof(batch_task) * (size_t)task_cap);
    if (e == cudaSuccess) e = cudaMalloc(&d_grids, sizeof(batch_grid_desc) * (size_t)grid_cap);
    if (e == cudaSuccess) e = cudaMalloc(&d_odd, (size_t)grid_cap);
    if (e == cudaSuccess) e = cudaMalloc(&d_counters, sizeof(unsigned) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_task_done, sizeof(unsigned) * (size_t)task_cap);
    if (e == cudaSuccess) e = cudaMallocHost(&h_tasks, sizeof(batch_task) * (size_t)task_cap);
    if (e == cudaSuccess) e = cudaMallocHost(&h_grids, sizeof(batch_grid_desc) * (size_t)grid_cap);
    if (e == cudaSuccess) e = cudaMallocHost(&h_odd, (size_t)grid_cap);
    if (e == cudaSuccess) e = cudaMallocHost(&h_misc, sizeof(unsigned) * 4);
    if (e == cudaSuccess) e = cudaMemset(d_odd, 0, (size_t)grid_cap);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return ecuda(e, "batch engine allocation");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    for (int k = 0; k < 2; ++k) {
        const void* fn = batch_kernel_for(k, kmax);
        int per_sm = 0;
        if (fn) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBatchKindWarps[k] * 32, 0);
        kind_blocks[k] = std::max(1, per_sm) * std::max(1, sms);
    }
    blocks = kind_blocks[kBatchBuiltin];
    return CB2_OK;
}

void batch_engine::release() {
    for (int k = 0; k < 2; ++k) {
        if (exec[k]) cudaGraphExecDestroy(exec[k]);
        if (graph[k]) cudaGraphDestroy(graph[k]);
    }
    if (cap_stream) cudaStreamDestroy(cap_stream);
    cudaFree(d_tasks);
    cudaFree(d_grids);
    cudaFree(d_odd);
    cudaFree(d_counters);
    cudaFree(d_task_done);
    cudaFreeHost(h_tasks);
    cudaFreeHost(h_grids);
    cudaFreeHost(h_odd);
    cudaFreeHost(h_misc);
    *this = batch_engine{};
}

// Fills h_tasks / h_grids / h_odd with the schedule of `items`.
int batch_engine::build(const std::vector<batch_item>& items, const batch_tiling& tiling) {
    const int n = (int)items.size();
    if (n > grid_cap) return efail(CB2_EINVAL, "batch holds more grids than its capacity");
    struct plan_t {
        std::vector<int> ks;  // K of each chunk
        int groups = 0, rows = 0, nsx = 1, nsy = 1;
    };
    std::vector<plan_t> plans((size_t)n);
    std::vector<int> order((size_t)n);
    kind = kBatchBuiltin;
    for (const batch_item& it : items)
        if (it.grid->g.automaton >= kNumBuiltin) kind = kBatchAll;
    // the kernel over every automaton runs chunks of at most kBatchKMax
    const int kcap = kind == kBatchAll ? std::min(kmax, kBatchKMax) : kmax;
    for (int i = 0; i < n; ++i) {
        const batch_item& it = items[(size_t)i];
        const cb2_grid* g = it.grid;
        plan_t& p = plans[(size_t)i];
        int64_t left = it.steps;
        const int kmain = std::min(kcap, tiling.temporal_steps > 0 ? tiling.temporal_steps : kcap);
        if (it.steps / kmain > INT_MAX) return efail(CB2_EINVAL, "too many generations for one batch run");
        while (left > 0) {
            int k = kmain;
            while (k > left) k /= 2;
            p.ks.push_back(k);
            left -= k;
        }
        const int wd = g->g.wd, h = g->g.h;
        const int rows = std::max(kmain, std::min(h, tiling.rows_for(g->g.automaton)));
        if (wd <= 16) {  // exact-wrap groups across the warp
            const int gmax = 32 / wd;
            p.rows = std::min(h, std::max((rows + gmax - 1) / gmax, 2 * kmain));
            p.groups = std::min(gmax, (h + p.rows - 1) / p.rows);
            p.nsx = 1;
            p.nsy = std::max(1, h / (p.rows * p.groups));
        } else {
            p.rows = rows;
            p.nsx = (wd + 29) / 30;
            p.nsy = std::max(1, h / rows);
        }
        if (p.nsx > 32767 || p.nsy > 32767) return efail(CB2_EINVAL, "grid too large for a batch task tiling");
        batch_grid_desc& d = h_grids[i];
        d.buf[0] = g->buf[it.cur];
        d.buf[1] = g->buf[it.cur ^ 1];
        d.plane_words = g->g.plane_words;
        d.wd = wd;
        d.h = h;
        d.automaton = g->g.automaton;
        d.t0 = it.t0;
        d.seed = it.seed;
        d.steps = it.steps;
        d.kmain = kmain;
        d.nfull = (int32_t)(it.steps / kmain);
        d.rem = (int32_t)(it.steps % kmain);
        h_odd[i] = (unsigned char)(p.ks.size() & 1);
        order[(size_t)i] = i;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return plans[(size_t)a].ks.size() > plans[(size_t)b].ks.size(); });
    std::vector<int> prev_base((size_t)n, -1);
    ntasks = 0;
    cells_per_run = 0;
    struct slot_t {
        double progress;
        int i, c;
    };
    std::vector<slot_t> slots;
    for (int i : order)
        for (int c = 0; c < (int)plans[(size_t)i].ks.size(); ++c)
            slots.push_back(slot_t{(c + 0.5) / (double)plans[(size_t)i].ks.size(), i, c});
    std::stable_sort(slots.begin(), slots.end(),
                     [](const slot_t& x, const slot_t& y) { return x.progress < y.progress; });
    for (const slot_t& sl : slots) {
        const int i = sl.i, c = sl.c;
        {
            const plan_t& p = plans[(size_t)i];
            const int per_chunk = p.nsx * p.nsy;
            if (ntasks + per_chunk > task_cap) return efail(CB2_ENOMEM, "batch task list is full");
            const int base = ntasks;
            const int h = items[(size_t)i].grid->g.h;
            const int span = p.groups ? p.rows * p.groups : p.rows;
            // A last strip of at most 14 own words runs as row bands side by side
            // in the warp (band_geom): floor(32 / (own words + 2)) of them, so that
            // it fills the warp.  The bands split the tile's rows exactly, so a
            // full tile takes a band count that divides its height.
            const int rem_words = items[(size_t)i].grid->g.wd - 30 * (p.nsx - 1);
            const int band_max = p.groups ? 1 : 32 / (rem_words + 2);
            for (int ty = 0; ty < p.nsy; ++ty) {
                const int y0 = ty * span;
                const bool last = ty == p.nsy - 1;
                // the last tile row takes every remaining row
                const int tile = last ? h - y0 : span;
                const int rows = !last ? p.rows
                                 : p.groups ? (h - y0 + p.groups - 1) / p.groups
                                            : h - y0;
                int bands = std::min(band_max, tile);
                if (!last)
                    while (tile % bands) --bands;
                for (int tx = 0; tx < p.nsx; ++tx) {
                    const bool banded = tx == p.nsx - 1 && bands > 1;
                    batch_task& t = h_tasks[ntasks++];
                    t.grid = i;
                    t.chunk = c;
                    t.dep_base = prev_base[(size_t)i];
                    t.rows = banded ? (tile + bands - 1) / bands : rows;
                    t.k = (int16_t)p.ks[(size_t)c];
                    t.groups = (int16_t)(banded ? -bands : p.groups);
                    t.nsx = (int16_t)p.nsx;
                    t.nsy = (int16_t)p.nsy;
                    t.tx = (int16_t)tx;
                    t.ty = (int16_t)ty;
                    t.y0 = y0;
                }
            }
            prev_base[(size_t)i] = base;
            const cb2_grid* g = items[(size_t)i].grid;
            cells_per_run += (double)g->g.x_size * g->g.y_size * p.ks[(size_t)c];
        }
    }
    ngrids = n;
    if (kind == kBatchAll && !generic_batch_kernel())
        return efail(CB2_EINVAL, "the library was built without the lowered DSL automata");
    blocks = kind_blocks[kind];
    return CB2_OK;
}

int batch_engine::upload(cudaStream_t s) {
    h_misc[0] = (unsigned)ntasks;
    h_misc[2] = (unsigned)ngrids;
    cudaError_t e = cudaMemcpyAsync(d_tasks, h_tasks, sizeof(batch_task) * (size_t)ntasks, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_grids, h_grids, sizeof(batch_grid_desc) * (size_t)ngrids, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_odd, h_odd, (size_t)ngrids, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_counters + 3, h_misc, sizeof(unsigned), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_counters + 2, h_misc + 2, sizeof(unsigned), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return ecuda(e, "batch task upload");
    return CB2_OK;
}

int batch_engine::capture(int k) {
    if (k != kBatchBuiltin && k != kBatchAll) return efail(CB2_EINVAL, "unknown batch kernel kind");
    if (exec[k]) return CB2_OK;
    const void* fn = batch_kernel_for(k, kmax);
    if (!fn) return efail(CB2_EINVAL, "the library was built without the lowered DSL automata");
    batch_args a;
    a.tasks = d_tasks;
    a.ntasks = d_counters + 3;
    a.grids = d_grids;
    a.task_done = d_task_done;
    a.head = d_counters;
    a.error = d_counters + 1;
    a.spin_limit = spin_limit;
    cudaError_t e = cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return ecuda(e, "batch graph capture");
    cudaMemsetAsync(d_counters, 0, sizeof(unsigned) * 2, cap_stream);  // head, error
    cudaMemsetAsync(d_task_done, 0, sizeof(unsigned) * (size_t)task_cap, cap_stream);
    void* args[] = {&a};
    cudaLaunchKernel(fn, dim3((unsigned)kind_blocks[k]), dim3(kBatchKindWarps[k] * 32), args, 0, cap_stream);
    const int nflip = grid_cap;
    batch_flip_kernel<<<(nflip + 255) / 256, 256, 0, cap_stream>>>(d_grids, d_odd, d_counters + 2);
    e = cudaStreamEndCapture(cap_stream, &graph[k]);
    if (e != cudaSuccess) return ecuda(e, "batch graph capture");
    e = cudaGraphInstantiate(&exec[k], graph[k], 0);
    if (e != cudaSuccess) return ecuda(e, "batch graph instantiate");
    return CB2_OK;
}

int batch_engine::launch(cudaStream_t s) {
    int rc = capture(kind);
    if (rc) return rc;
    cudaError_t e = cudaGraphLaunch(exec[kind], s);
    if (e != cudaSuccess) return ecuda(e, "batch graph launch");
    return CB2_OK;
}

int batch_engine::check(cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(h_misc + 1, d_counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return ecuda(e, "batch completion");
    if (h_misc[1])
        return efail(CB2_ETIMEOUT, "batch task " + std::to_string(h_misc[1] - 1) +
                                       " waited longer than its spin limit for the previous chunk of its grid");
    return CB2_OK;
}

int batch_engine::read_error_async(cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(h_misc + 1, d_counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return ecuda(e, "batch error read-back");
    return CB2_OK;
}

int batch_engine::error_seen() {
    if (h_misc[1])
        return efail(CB2_ETIMEOUT, "batch task " + std::to_string(h_misc[1] - 1) +
                                       " waited longer than its spin limit for the previous chunk of its grid");
    return CB2_OK;
}

} // namespace cb2

using namespace cb2;

struct cb2_batch {
    batch_engine eng;
    std::vector<batch_item> items;
    batch_tiling tiling;
    bool built = false;     // h_tasks holds the schedule of `items`
    bool uploaded = false;  // and the device has it
};

extern "C" {

int cb2_batch_create(cb2_grid* const* grids, const int64_t* steps, int n, const cb2_batch_opts* opts, cb2_batch** out) {
    if (!out || !grids || !steps || n <= 0) return efail(CB2_EINVAL, "null argument or empty batch");
    cb2_batch_opts o{0, 0, 0, -1};
    if (opts) o = *opts;
    if (o.temporal_steps && o.temporal_steps != 1 && o.temporal_steps != 2 && o.temporal_steps != 4 &&
        o.temporal_steps != 8 && o.temporal_steps != 16 && o.temporal_steps != 32)
        return efail(CB2_EINVAL, "batch temporal_steps must be 1, 2, 4, 8, 16 or 32");
    auto* b = new cb2_batch();
    // Defaults measured on the batched workload (4096 mixed network grids):
    // chunks of 8 generations and 256-row tiles 20.5 Tcell/s, 16 and 512 rows
    // 21.4, 32 and 512 rows 23.5, 32 and 768 rows 23.9, 32 and 1024 rows 22.7.
    b->tiling.temporal_steps = o.temporal_steps ? o.temporal_steps : kBatchDefaultK;
    b->tiling.tile_rows = o.tile_rows > 0 ? o.tile_rows : kBatchDefaultRows;
    b->tiling.lowered_tile_rows = o.tile_rows > 0 ? o.tile_rows : 64;
    bool lowered = false;  // a lowered DSL automaton caps every chunk of the batch at kBatchKMax
    for (int i = 0; i < n; ++i) lowered = lowered || (grids[i] && grids[i]->g.automaton >= kNumBuiltin);
    const int kchunk = lowered ? std::min(b->tiling.temporal_steps, kBatchKMax) : b->tiling.temporal_steps;
    int64_t est = 0;
    for (int i = 0; i < n; ++i) {
        if (!grids[i] || steps[i] < 0) {
            delete b;
            return efail(CB2_EINVAL, "null grid or negative steps in batch");
        }
        b->items.push_back(batch_item{grids[i], steps[i], grids[i]->cur, grids[i]->time_step, grids[i]->seed});
        const cb2_grid* g = grids[i];
        const int64_t chunks = steps[i] / std::max(1, kchunk) + 6;
        const int64_t rows = std::max<int64_t>(1, std::min<int64_t>(g->g.h, b->tiling.rows_for(g->g.automaton)));
        const int64_t per_chunk =
            g->g.wd <= 16 ? (g->g.h + 1) / 2 + 1 : ((g->g.h + rows - 1) / rows) * ((g->g.wd + 29) / 30);
        est += chunks * per_chunk;
    }
    if (est > INT_MAX / 2) {
        delete b;
        return efail(CB2_EINVAL, "batch too large for one task list");
    }
    int rc = b->eng.init((int)est, n, b->tiling.temporal_steps, o.spin_limit);
    if (!rc) rc = b->eng.build(b->items, b->tiling);
    if (!rc && o.stall_task >= 0 && o.stall_task < b->eng.ntasks) {
        // test hook: a dependency nothing satisfies -- the task waits on its own flag
        batch_task& t = b->eng.h_tasks[o.stall_task];
        t.dep_base = o.stall_task - (t.ty * t.nsx + t.tx);
    }
    b->built = rc == CB2_OK;
    if (rc) {
        b->eng.release();
        delete b;
        return rc;
    }
    *out = b;
    return CB2_OK;
}

int cb2_batch_destroy(cb2_batch* b) {
    if (!b) return CB2_OK;
    b->eng.release();
    delete b;
    return CB2_OK;
}

int cb2_batch_run(cb2_batch* b, void* stream) {
    if (!b) return efail(CB2_EINVAL, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    for (batch_item& it : b->items)
        if (it.grid->cur != it.cur || it.grid->time_step != it.t0 || it.grid->seed != it.seed) {
            // the grid was advanced, re-uploaded, re-timed or re-seeded outside the batch
            b->built = false;
            it.cur = it.grid->cur;
            it.t0 = it.grid->time_step;
            it.seed = it.grid->seed;
        }
    if (!b->built) {
        // the pinned task list may still feed an earlier upload on this stream
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return ecuda(e, "batch rebuild");
        int rc = b->eng.build(b->items, b->tiling);
        if (rc) return rc;
        b->built = true;
        b->uploaded = false;
    }
    if (!b->uploaded) {
        int rc = b->eng.upload(s);
        if (rc) return rc;
        b->uploaded = true;
    }
    int rc = b->eng.launch(s);
    if (rc) return rc;
    for (batch_item& it : b->items) {
        if (b->eng.h_odd[&it - b->items.data()]) {
            it.grid->cur ^= 1;
            it.cur = it.grid->cur;
        }
        it.grid->time_step += it.steps;
        it.t0 = it.grid->time_step;  // as batch_flip_kernel advances the device copy
    }
    return CB2_OK;
}

int cb2_batch_wait(cb2_batch* b, void* stream) {
    if (!b) return efail(CB2_EINVAL, "null batch");
    return b->eng.check((cudaStream_t)stream);
}

int cb2_batch_run_per_grid(cb2_batch* b, void* stream) {
    if (!b) return efail(CB2_EINVAL, "null batch");
    for (batch_item& it : b->items) {
        int rc = cb2_grid_run(it.grid, it.steps, nullptr, stream);
        if (rc) return rc;
    }
    return CB2_OK;
}

int cb2_batch_info(const cb2_batch* b, int64_t* tasks, double* cell_updates, int* persistent_ctas) {
    if (!b) return efail(CB2_EINVAL, "null batch");
    if (tasks) *tasks = b->eng.ntasks;
    if (cell_updates) *cell_updates = b->eng.cells_per_run;
    if (persistent_ctas) *persistent_ctas = b->eng.blocks;
    return CB2_OK;
}

} // extern "C"
