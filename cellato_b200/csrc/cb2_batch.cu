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
#include "cellato_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "cb2_batch.h"
#include "cb2_internal.h"
#include "cb2_pipe.cuh"
#include "cb2_rules.cuh"

namespace cb2 {

constexpr int kBatchWarps = 4;   // warps of a CTA: one task per CTA, its levels split over them
constexpr int kBatchPlanes = 3;  // the hand-written networks' largest P
constexpr int kBatchRows = 4;    // rows each warp passes on per barrier (2: 18.3, 4: 19.1 Tcell/s)
// Shared memory of the largest task pipeline (K = 8 over the 4 warps, P = 3):
// the input ring plus two four-row hand-off slots per warp boundary.
constexpr int kBatchSmemWords = (kRingDepth + 2 * kBatchRows * (kBatchWarps - 1)) * kBatchPlanes * 32;

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

// One chunk of K generations of one task on the whole CTA: the level pipeline
// of pipe_run_rows with the K levels split over the warps (K = 8: two levels
// per warp, K = 4: one), which divides a task's latency -- and with it the
// length of a grid's chain of chunks -- by the number of warps.  Chunks
// shorter than the CTA (K = 2, 1) leave warps idle at the barriers.
template <class R, int K>
__device__ __forceinline__ void batch_run_task(const strip_task& t, const lane_geom<1>& geom, uint32_t* smem) {
    constexpr int L = K >= kBatchWarps ? K / kBatchWarps : 1;
    constexpr int W = K / L;
    static_assert(pipe_rows_smem_words<R, K, 1, L, kRingDepth, kBatchRows>() <= kBatchSmemWords,
                  "task pipeline larger than the CTA's shared memory");
    if ((int)(threadIdx.x >> 5) < W)
        pipe_run_rows<R, K, 1, L, kRingDepth, kBatchRows>(t, geom, smem);
    else
        pipe_rows_idle<K, L, kBatchRows>(t);
}

template <class R, int KMAX>
__device__ __forceinline__ void batch_run_rule(const strip_task& t, int k, const lane_geom<1>& geom, uint32_t* smem) {
    switch (k) {
    case 1: batch_run_task<R, 1>(t, geom, smem); break;
    case 2: batch_run_task<R, 2>(t, geom, smem); break;
    case 4: batch_run_task<R, 4>(t, geom, smem); break;
    default:
        if constexpr (KMAX >= 8) batch_run_task<R, 8>(t, geom, smem);
        break;
    }
}

template <int KMAX>
__global__ void __launch_bounds__(kBatchWarps * 32) batch_kernel(batch_args a) {
    __shared__ __align__(16) uint32_t smem[kBatchSmemWords];
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
        st.t0 = 0;  // the hand-written networks read neither time, seed nor global rows
        st.seed = 0;
        st.y_global0 = 0;
        st.global_h = gd.h;
        st.wd = gd.wd;
        st.h = gd.h;
        lane_geom<1> geom;
        st.y0 = task.y0;
        st.ny = task.rows;
        if (task.groups) {
            st.x0 = 0;
            st.nx = gd.wd;
            geom = group_geom(st, task.groups, lane);
        } else {
            st.x0 = task.tx * 30;
            st.nx = min(30, gd.wd - st.x0);
            geom = strip_geom<1>(st, lane);
        }
        switch (gd.automaton) {
        case 0: batch_run_rule<game_of_life, KMAX>(st, task.k, geom, smem); break;
        case 1: batch_run_rule<wire, KMAX>(st, task.k, geom, smem); break;
        default: batch_run_rule<excitable, KMAX>(st, task.k, geom, smem); break;
        }
        __threadfence();  // this thread's stores are visible GPU-wide before the flag
        __syncthreads();  // every warp's stores are done; smem and s_task are free again
        if (threadIdx.x == 0) atomicExch(a.task_done + t, 1u);
    }
}

// After a run, a grid that took an odd number of chunks holds its result in
// buffer 1: swap so that buffer 0 is again the current generation.
__global__ void batch_flip_kernel(batch_grid_desc* grids, const unsigned char* odd, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && odd[i]) {
        uint32_t* t = grids[i].buf[0];
        grids[i].buf[0] = grids[i].buf[1];
        grids[i].buf[1] = t;
    }
}

static const void* batch_kernel_for(int kmax) {
    return kmax >= 8 ? (const void*)batch_kernel<8> : (const void*)batch_kernel<4>;
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
    kmax = kmax_ >= 8 ? 8 : 4;
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
    const void* fn = batch_kernel_for(kmax);
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBatchWarps * 32, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    blocks = std::max(1, per_sm) * std::max(1, sms);
    return CB2_OK;
}

void batch_engine::release() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
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
    for (int i = 0; i < n; ++i) {
        const batch_item& it = items[(size_t)i];
        const cb2_grid* g = it.grid;
        plan_t& p = plans[(size_t)i];
        int64_t left = it.steps;
        const int kmain = std::min(kmax, tiling.temporal_steps > 0 ? tiling.temporal_steps : kmax);
        while (left > 0) {
            int k = kmain;
            while (k > left) k /= 2;
            p.ks.push_back(k);
            left -= k;
        }
        const int wd = g->g.wd, h = g->g.h;
        const int rows = std::max(kmain, std::min(h, tiling.tile_rows));
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
        d.pad = 0;
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
            for (int ty = 0; ty < p.nsy; ++ty) {
                const int y0 = ty * span;
                const bool last = ty == p.nsy - 1;
                // the last tile row takes every remaining row
                const int rows = !last ? p.rows
                                 : p.groups ? (h - y0 + p.groups - 1) / p.groups
                                            : h - y0;
                for (int tx = 0; tx < p.nsx; ++tx) {
                    batch_task& t = h_tasks[ntasks++];
                    t.grid = i;
                    t.chunk = c;
                    t.dep_base = prev_base[(size_t)i];
                    t.rows = rows;
                    t.k = (int16_t)p.ks[(size_t)c];
                    t.groups = (int16_t)p.groups;
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
    return CB2_OK;
}

int batch_engine::upload(cudaStream_t s) {
    h_misc[0] = (unsigned)ntasks;
    cudaError_t e = cudaMemcpyAsync(d_tasks, h_tasks, sizeof(batch_task) * (size_t)ntasks, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_grids, h_grids, sizeof(batch_grid_desc) * (size_t)ngrids, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_odd, h_odd, (size_t)ngrids, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_counters + 3, h_misc, sizeof(unsigned), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return ecuda(e, "batch task upload");
    return CB2_OK;
}

int batch_engine::capture() {
    if (exec) return CB2_OK;
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
    cudaMemsetAsync(d_counters, 0, sizeof(unsigned) * 3, cap_stream);
    cudaMemsetAsync(d_task_done, 0, sizeof(unsigned) * (size_t)task_cap, cap_stream);
    void* args[] = {&a};
    cudaLaunchKernel(batch_kernel_for(kmax), dim3((unsigned)blocks), dim3(kBatchWarps * 32), args, 0, cap_stream);
    const int nflip = grid_cap;
    batch_flip_kernel<<<(nflip + 255) / 256, 256, 0, cap_stream>>>(d_grids, d_odd, nflip);
    e = cudaStreamEndCapture(cap_stream, &graph);
    if (e != cudaSuccess) return ecuda(e, "batch graph capture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) return ecuda(e, "batch graph instantiate");
    return CB2_OK;
}

int batch_engine::launch(cudaStream_t s) {
    int rc = capture();
    if (rc) return rc;
    cudaError_t e = cudaGraphLaunch(exec, s);
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
        o.temporal_steps != 8)
        return efail(CB2_EINVAL, "batch temporal_steps must be 1, 2, 4 or 8");
    auto* b = new cb2_batch();
    b->tiling.temporal_steps = o.temporal_steps ? o.temporal_steps : 8;
    b->tiling.tile_rows = o.tile_rows > 0 ? o.tile_rows : 256;
    int64_t est = 0;
    for (int i = 0; i < n; ++i) {
        if (!grids[i] || steps[i] < 0) {
            delete b;
            return efail(CB2_EINVAL, "null grid or negative steps in batch");
        }
        if (grids[i]->g.automaton >= kNumBuiltin) {
            delete b;
            return efail(CB2_EINVAL, std::string("the batch kernel runs game-of-life, wire and excitable; '") +
                                         name_of(grids[i]->g.automaton) + "' advances with cb2_grid_run");
        }
        b->items.push_back(batch_item{grids[i], steps[i], grids[i]->cur});
        const cb2_grid* g = grids[i];
        const int64_t chunks = steps[i] / std::max(1, b->tiling.temporal_steps) + 4;
        const int64_t rows = std::max<int64_t>(1, std::min<int64_t>(g->g.h, b->tiling.tile_rows));
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
        if (it.grid->cur != it.cur) {  // the grid was advanced or re-uploaded outside the batch
            b->built = false;
            it.cur = it.grid->cur;
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
