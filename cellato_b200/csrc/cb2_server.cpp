// cb2_server.cpp -- the serving loop: continuous batching of simulation
// requests on one GPU.
//
// Clients submit requests (automaton, size, generations, seeded or host
// input) from any thread.  One server thread owns the GPU work:
//
//   admit   requests leave the FIFO queue while their double-buffered bit
//           planes fit in the device-memory budget and a slot is free; their
//           state is allocated from a stream-ordered pool and initialised on
//           the device.
//   round   every active request advances up to chunk_steps generations in
//           one replay of a batch engine's graph (cb2_batch.cu): one
//           persistent kernel over all their tasks (the kernel over every
//           automaton when the round holds a lowered DSL rule, with each
//           request's generation and seed).  Requests of at least
//           direct_cells cells instead advance through the single-grid strip
//           kernels (cb2_grid_run's plan: up to 32 generations per HBM round
//           trip, one CTA of several warps per strip) on side streams (each
//           request keeps one, so its passes stay in order; several requests'
//           passes run side by side), so their passes fill the SMs that the
//           batch kernel's tail leaves idle; a round is retired when its work
//           on every stream has passed.  Optionally (round_cells)
//           a request's share is sized so that a round holds about that many
//           cell-updates -- more generations for small grids, fewer for big
//           ones -- still capped at chunk_steps.
//   retire  a request's last round is followed, in stream order, by its
//           16-number checksum (and, if asked, its cells); when the round's
//           event has passed, the request is marked done, its memory goes
//           back to the pool and its waiters wake.
//
// Two engines alternate, so the host plans and uploads round r+1 while the
// GPU runs round r; requests that arrive meanwhile are admitted at the next
// round, and their work overlaps on the device with the requests already in
// flight.  State stays resident between rounds.  With per_request = 1 the
// same loop runs the plain path instead: one request at a time, its
// generations launched as one sequence of strip passes with the library's
// default plan (cb2_grid_run's path), which is what a traverser per request
// does.
//
// Failures are per request: an allocation that fails (or the test hook
// fail_alloc_at) fails that request with CB2_ENOMEM; a round whose bounded
// wait ran out fails the requests of that round with CB2_ETIMEOUT.  Nothing
// in the loop blocks the GPU.
#include "cellato_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cb2_batch.h"
#include "cb2_internal.h"

namespace cb2 {
namespace {

using clock_t_ = std::chrono::steady_clock;

constexpr int kDirectStreams = 4;  // side streams for the strip passes of large requests

struct request_state {
    int64_t id = 0;
    int side = 0;  // side stream of a large request
    cb2_request req{};
    std::vector<uint64_t> thr;
    int state = CB2_REQ_QUEUED;
    int error = 0;
    std::string message;
    int64_t done_steps = 0;
    double submit_s = 0, admit_s = 0, done_s = 0;
    uint64_t checksum[16] = {};
    size_t bytes = 0;      // device bytes of the double buffer
    cb2_grid grid{};       // device state while active
    int64_t planned = 0;   // generations queued on the GPU so far
    int slot = -1;         // checksum slot
    bool settled = false;  // finished (done or failed)
};

// A round queued on the GPU.
struct round_rec {
    int engine = 0;
    bool batched = false;  // the round launched the engine's batch kernel
    cudaEvent_t done = nullptr;         // main stream: batch kernel and its results
    cudaEvent_t done_direct[kDirectStreams] = {};  // side streams: strip passes and their results
    std::vector<request_state*> members;
    std::vector<request_state*> finishing;
    double cells = 0;
};

} // namespace

struct server_impl {
    cb2_server_opts opts{};
    int device = 0;
    clock_t_::time_point t0;
    cudaStream_t stream = nullptr;
    cudaStream_t direct[kDirectStreams] = {};  // strip passes of the large requests
    cudaEvent_t ev_fork = nullptr;  // main stream -> side streams, after a large request's initialisation
    bool direct_fork_needed = false;
    int next_side = 0;
    cudaMemPool_t pool = nullptr;
    unsigned long long* d_sums = nullptr;  // 16 checksum sums, then the conversion flag
    unsigned long long* h_sums = nullptr;
    size_t rot = 0;  // first request of the next round
    batch_engine engs[2];
    bool engine_ready[2] = {false, false};
    int next_engine = 0;
    batch_tiling tiling;
    std::deque<round_rec> inflight;
    std::vector<cudaEvent_t> spare_events;
    unsigned long long* d_slots = nullptr;  // 16 sums per checksum slot
    unsigned long long* h_slots = nullptr;  // pinned mirror
    std::vector<int> free_slots;

    std::mutex mu;
    std::condition_variable cv_work;  // the server thread waits for requests
    std::condition_variable cv_done;  // clients wait for completions
    std::map<int64_t, std::unique_ptr<request_state>> reqs;
    std::deque<request_state*> queue;  // submitted, not admitted
    std::vector<request_state*> active;
    int64_t next_id = 1;
    size_t used_bytes = 0;
    long long allocs = 0;
    bool stop = false;
    cb2_server_stats stats{};
    std::thread thread;

    double now() const { return std::chrono::duration<double>(clock_t_::now() - t0).count(); }

    int alloc_grid(request_state* r);
    void free_grid(request_state* r);
    void finish(request_state* r, int error, const std::string& msg);
    void loop();
    void launch_round();
    void retire_round(round_rec& rr);
    void run_one(request_state* r);
    bool admit_locked(std::vector<request_state*>& newly);
    int init_grid(request_state* r);
    int retire(request_state* r);
    bool is_direct(const request_state* r) const {
        return opts.direct_cells > 0 && (double)r->req.x_size * (double)r->req.y_size >= (double)opts.direct_cells;
    }
    cudaError_t enqueue_result(request_state* r, cudaStream_t s);
    cudaEvent_t take_event();
    bool round_passed(const round_rec& rr) {
        if (cudaEventQuery(rr.done) != cudaSuccess) return false;
        for (cudaEvent_t ev : rr.done_direct)
            if (ev && cudaEventQuery(ev) != cudaSuccess) return false;
        return true;
    }
    void sync_round(const round_rec& rr) {
        cudaEventSynchronize(rr.done);
        for (cudaEvent_t ev : rr.done_direct)
            if (ev) cudaEventSynchronize(ev);
    }
    void sync_direct() {
        for (cudaStream_t s : direct)
            if (s) cudaStreamSynchronize(s);
    }
};

cudaEvent_t server_impl::take_event() {
    if (spare_events.empty()) {
        cudaEvent_t ev = nullptr;
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        return ev;
    }
    cudaEvent_t ev = spare_events.back();
    spare_events.pop_back();
    return ev;
}

int server_impl::alloc_grid(request_state* r) {
    ++allocs;
    if (opts.fail_alloc_at > 0 && allocs == opts.fail_alloc_at) {
        set_error("injected allocation failure");
        return CB2_ENOMEM;
    }
    grid_geom g;
    int rc = make_geom(r->req.automaton, r->req.x_size, r->req.y_size, &g);
    if (rc) return rc;
    const size_t half = (size_t)g.planes * (size_t)g.plane_words * 4;
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, 2 * half, pool, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("request state allocation: ") + cudaGetErrorString(e));
        return CB2_ENOMEM;
    }
    r->grid.g = g;
    r->grid.buf[0] = (uint32_t*)p;
    r->grid.buf[1] = (uint32_t*)((char*)p + half);
    r->grid.cur = 0;
    r->grid.time_step = 0;
    return CB2_OK;
}

void server_impl::free_grid(request_state* r) {
    if (r->grid.buf[0]) cudaFreeAsync(r->grid.buf[0], stream);
    r->grid.buf[0] = r->grid.buf[1] = nullptr;
}

int server_impl::init_grid(request_state* r) {
    const grid_geom& g = r->grid.g;
    cudaError_t e;
    if (r->req.host_cells) {
        // one uint8 dictionary index per cell, staged in a pool buffer and packed
        const size_t n = (size_t)g.x_size * (size_t)g.y_size;
        unsigned* flag = (unsigned*)(d_sums + 16);
        void* tmp = nullptr;
        e = cudaMallocFromPoolAsync(&tmp, n, pool, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, r->req.host_cells, n, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(unsigned), stream);
        if (e == cudaSuccess) e = launch_pack_cells(g, tmp, 1, r->grid.buf[0], flag, stream);
        if (tmp) cudaFreeAsync(tmp, stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h_sums + 16, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess && (unsigned)h_sums[16]) {
            set_error("State not found in dictionary (a cell value exceeds the automaton's states)");
            return CB2_ESTATE;
        }
    } else {
        e = launch_fill_random(g, r->grid.buf[0], r->req.seed, r->thr.data(), (int)r->thr.size(), stream);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("request input: ") + cudaGetErrorString(e));
        return CB2_ECUDA;
    }
    return CB2_OK;
}

// Checksum (and result copy) of a finished request; synchronises the stream.
int server_impl::retire(request_state* r) {
    const grid_geom& g = r->grid.g;
    const uint32_t* cur = r->grid.buf[r->grid.cur];
    cudaError_t e = cudaMemsetAsync(d_sums, 0, 16 * sizeof(unsigned long long), stream);
    if (e == cudaSuccess) e = launch_checksum(g, cur, nullptr, 0, d_sums, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_sums, d_sums, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && r->req.host_result) {
        const size_t n = (size_t)g.x_size * (size_t)g.y_size;
        void* tmp = nullptr;
        e = cudaMallocFromPoolAsync(&tmp, n, pool, stream);
        if (e == cudaSuccess) e = launch_unpack_cells(g, cur, tmp, 1, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(r->req.host_result, tmp, n, cudaMemcpyDeviceToHost, stream);
        if (tmp) cudaFreeAsync(tmp, stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("request result: ") + cudaGetErrorString(e));
        return CB2_ECUDA;
    }
    for (int i = 0; i < 16; ++i) r->checksum[i] = h_sums[i];
    return CB2_OK;
}

void server_impl::finish(request_state* r, int error, const std::string& msg) {
    if (r->settled) return;
    r->settled = true;
    free_grid(r);
    if (r->slot >= 0) {
        free_slots.push_back(r->slot);
        r->slot = -1;
    }
    std::lock_guard<std::mutex> lock(mu);
    used_bytes -= r->bytes;
    r->state = error ? CB2_REQ_FAILED : CB2_REQ_DONE;
    r->error = error;
    r->message = msg;
    r->done_s = now();
    if (error)
        ++stats.failed;
    else
        ++stats.completed;
    cv_done.notify_all();
}

// Moves queued requests to `newly` while slots and budget allow (FIFO).
bool server_impl::admit_locked(std::vector<request_state*>& newly) {
    const int max_active = opts.per_request ? 1 : opts.max_active;
    while (!queue.empty() && (int)(active.size() + newly.size()) < max_active) {
        request_state* r = queue.front();
        if (used_bytes + r->bytes > opts.memory_budget) break;
        queue.pop_front();
        used_bytes += r->bytes;
        r->state = CB2_REQ_ACTIVE;
        r->admit_s = now();
        newly.push_back(r);
    }
    return !newly.empty();
}

void server_impl::run_one(request_state* r) {
    uint32_t* const bufs[2] = {r->grid.buf[0], r->grid.buf[1]};
    int res = 0;
    int rc = run_chunks(r->grid.g, bufs, 0, r->req.steps, nullptr, stream, &res, 0, r->req.seed);  // the default plan
    if (rc) {
        finish(r, rc, cb2_last_error());
        return;
    }
    r->grid.cur = res;
    r->done_steps = r->req.steps;
    rc = retire(r);
    {
        std::lock_guard<std::mutex> lock(mu);
        stats.cell_updates += (double)r->req.x_size * r->req.y_size * r->req.steps;
        ++stats.rounds;
    }
    finish(r, rc, rc ? cb2_last_error() : "");
}

// Checksum (and, if asked, cells) of a request whose last generation is
// queued on `s`, into its slot; read by retire_round after the round's event.
cudaError_t server_impl::enqueue_result(request_state* r, cudaStream_t s) {
    const grid_geom& g = r->grid.g;
    const uint32_t* cur = r->grid.buf[r->grid.cur];
    unsigned long long* sums = d_slots + 16 * (size_t)r->slot;
    cudaError_t ce = cudaMemsetAsync(sums, 0, 16 * sizeof(unsigned long long), s);
    if (ce == cudaSuccess) ce = launch_checksum(g, cur, nullptr, 0, sums, s);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(h_slots + 16 * (size_t)r->slot, sums, 16 * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess && r->req.host_result) {
        const size_t cells = (size_t)g.x_size * (size_t)g.y_size;
        void* tmp = nullptr;
        ce = cudaMallocFromPoolAsync(&tmp, cells, pool, s);
        if (ce == cudaSuccess) ce = launch_unpack_cells(g, cur, tmp, 1, s);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(r->req.host_result, tmp, cells, cudaMemcpyDeviceToHost, s);
        if (tmp) cudaFreeAsync(tmp, s);
    }
    return ce;
}

void server_impl::launch_round() {
    const int e = next_engine;
    // Shares: about round_cells cell-updates over the requests with work left.
    std::vector<request_state*> todo;
    for (request_state* r : active)
        if (r->planned < r->req.steps) todo.push_back(r);
    if (todo.empty()) return;
    const int K = tiling.temporal_steps;
    const double share = opts.round_cells > 0 ? opts.round_cells / (double)todo.size() : 0.0;
    std::vector<batch_item> items;
    std::vector<request_state*> in_round;  // batch kernel members, in item order
    std::vector<std::pair<request_state*, int64_t>> direct_items;
    const size_t n = todo.size();
    for (size_t j = 0; j < n; ++j) {
        request_state* r = todo[(rot + j) % n];
        const int64_t left = r->req.steps - r->planned;
        const double cells = (double)r->req.x_size * (double)r->req.y_size;
        int64_t steps = opts.chunk_steps;
        if (share > 0) {  // clamp in floating point: the quotient can exceed any integer
            const double fit = std::min(share / cells, (double)opts.chunk_steps);
            steps = std::max<int64_t>((int64_t)fit / K * K, K);
        }
        steps = std::min<int64_t>(steps, left);
        if (is_direct(r)) {
            direct_items.push_back({r, steps});
        } else {
            // generations already planned and the request's seed, for time- and seed-dependent rules
            items.push_back(batch_item{&r->grid, steps, r->grid.cur, r->planned, r->req.seed});
            in_round.push_back(r);
        }
    }
    rot = n ? (rot + 1) % n : 0;
    int rc = CB2_OK;
    if (!items.empty() && !engine_ready[e]) {
        rc = engs[e].init(opts.task_capacity, opts.max_active, tiling.temporal_steps, opts.spin_limit);
        if (rc) {
            const std::string msg = cb2_last_error();
            for (request_state* r : in_round) finish(r, rc, msg);
            active.erase(std::remove_if(active.begin(), active.end(), [](request_state* r) { return r->settled; }),
                         active.end());
            return;
        }
        engine_ready[e] = true;
    }
    batch_engine& eng = engs[e];
    if (!items.empty()) {
        rc = eng.build(items, tiling);
        while (rc == CB2_ENOMEM && items.size() > 1) {  // too many tasks: the rest wait for the next round
            items.pop_back();
            in_round.pop_back();
            rc = eng.build(items, tiling);
        }
    }
    round_rec rr;
    rr.engine = e;
    rr.members = in_round;
    for (auto& d : direct_items) rr.members.push_back(d.first);
    // A large request's passes follow each other on its side stream; the side
    // streams wait for the main stream only after a large request's state was
    // initialised there.
    cudaError_t ce = cudaSuccess;
    if (!rc && !direct_items.empty() && direct_fork_needed) {
        direct_fork_needed = false;
        ce = cudaEventRecord(ev_fork, stream);
        for (int i = 0; i < kDirectStreams && ce == cudaSuccess; ++i) ce = cudaStreamWaitEvent(direct[i], ev_fork, 0);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            rc = CB2_ECUDA;
            set_error(std::string("round fork: ") + cudaGetErrorString(ce));
        }
    }
    if (!rc && !items.empty()) {
        rc = eng.upload(stream);
        if (!rc) rc = eng.launch(stream);
        if (!rc) rc = eng.read_error_async(stream);
        if (!rc) {
            rr.batched = true;
            std::lock_guard<std::mutex> lock(mu);
            stats.tasks += eng.ntasks;
        }
    }
    if (!rc) {
        for (size_t i = 0; i < in_round.size(); ++i) {
            request_state* r = in_round[i];
            if (eng.h_odd[i]) r->grid.cur ^= 1;
            r->planned += items[i].steps;
            rr.cells += (double)r->req.x_size * r->req.y_size * items[i].steps;
            if (r->planned < r->req.steps) continue;
            rr.finishing.push_back(r);  // last round of r: checksum (and cells) follow in stream order
            ce = enqueue_result(r, stream);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                rc = CB2_ECUDA;
                set_error(std::string("request result: ") + cudaGetErrorString(ce));
                break;
            }
        }
    }
    if (!rc && !direct_items.empty()) {
        bool used[kDirectStreams] = {};
        for (auto& d : direct_items) {
            request_state* r = d.first;
            cudaStream_t side = direct[r->side];
            used[r->side] = true;
            uint32_t* const bufs[2] = {r->grid.buf[0], r->grid.buf[1]};
            int res = r->grid.cur;
            rc = run_chunks(r->grid.g, bufs, r->grid.cur, d.second, nullptr, side, &res, r->planned, r->req.seed);
            if (rc) break;
            r->grid.cur = res;
            r->planned += d.second;
            rr.cells += (double)r->req.x_size * r->req.y_size * d.second;
            if (r->planned < r->req.steps) continue;
            rr.finishing.push_back(r);
            ce = enqueue_result(r, side);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                rc = CB2_ECUDA;
                set_error(std::string("request result: ") + cudaGetErrorString(ce));
                break;
            }
        }
        for (int i = 0; i < kDirectStreams && !rc; ++i) {
            if (!used[i]) continue;
            rr.done_direct[i] = take_event();
            ce = cudaEventRecord(rr.done_direct[i], direct[i]);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                rc = CB2_ECUDA;
                set_error(std::string("round event: ") + cudaGetErrorString(ce));
            }
        }
    }
    if (!rc) {
        rr.done = take_event();
        ce = cudaEventRecord(rr.done, stream);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            rc = CB2_ECUDA;
            set_error(std::string("round event: ") + cudaGetErrorString(ce));
        }
    }
    if (rc) {
        // A failed launch: the round's requests fail, the rest go on.
        sync_direct();
        cudaStreamSynchronize(stream);
        const std::string msg = cb2_last_error();
        for (request_state* r : rr.members) finish(r, rc, msg);
        active.erase(std::remove_if(active.begin(), active.end(), [](request_state* r) { return r->settled; }),
                     active.end());
        if (rr.done) spare_events.push_back(rr.done);
        for (cudaEvent_t ev : rr.done_direct)
            if (ev) spare_events.push_back(ev);
        return;
    }
    if (rr.batched) next_engine ^= 1;
    inflight.push_back(std::move(rr));
}

void server_impl::retire_round(round_rec& rr) {
    const int rc = rr.batched ? engs[rr.engine].error_seen() : CB2_OK;
    spare_events.push_back(rr.done);
    for (cudaEvent_t ev : rr.done_direct)
        if (ev) spare_events.push_back(ev);
    if (rc) {
        // a bounded wait ran out: the round's requests hold no valid state
        const std::string msg = cb2_last_error();
        for (request_state* r : rr.members) finish(r, rc, msg);
    } else {
        for (request_state* r : rr.finishing) {
            for (int i = 0; i < 16; ++i) r->checksum[i] = h_slots[16 * (size_t)r->slot + i];
            r->done_steps = r->req.steps;
            finish(r, CB2_OK, "");
        }
        for (request_state* r : rr.members)
            if (!r->settled) r->done_steps = r->planned;
    }
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!rc) stats.cell_updates += rr.cells;
        ++stats.rounds;
    }
    active.erase(std::remove_if(active.begin(), active.end(), [](request_state* r) { return r->settled; }),
                 active.end());
}

void server_impl::loop() {
    cudaSetDevice(device);
    for (;;) {
        std::vector<request_state*> newly;
        {
            std::unique_lock<std::mutex> lock(mu);
            if (inflight.empty() && active.empty())
                cv_work.wait(lock, [&] { return stop || !queue.empty(); });
            if (stop) break;
            admit_locked(newly);
        }
        for (request_state* r : newly) {
            if (!free_slots.empty()) {
                r->slot = free_slots.back();
                free_slots.pop_back();
            }
            int rc = alloc_grid(r);
            if (!rc) rc = init_grid(r);
            if (rc) {
                finish(r, rc, cb2_last_error());
                continue;
            }
            if (is_direct(r)) {
                direct_fork_needed = true;
                r->side = next_side;
                next_side = (next_side + 1) % kDirectStreams;
            }
            if (opts.per_request)
                run_one(r);
            else
                active.push_back(r);
        }
        if (opts.per_request) continue;
        while (!inflight.empty() && round_passed(inflight.front())) {
            retire_round(inflight.front());
            inflight.pop_front();
        }
        bool work = false;
        for (request_state* r : active)
            if (r->planned < r->req.steps) {
                work = true;
                break;
            }
        if (work && inflight.size() < 2) {
            const double t_plan = now();
            launch_round();
            const double dt = now() - t_plan;
            std::lock_guard<std::mutex> lock(mu);
            stats.plan_s += dt;
            continue;
        }
        if (!inflight.empty()) {
            const double t_wait = now();
            sync_round(inflight.front());
            {
                const double dt = now() - t_wait;
                std::lock_guard<std::mutex> lock(mu);
                stats.wait_s += dt;
            }
            retire_round(inflight.front());
            inflight.pop_front();
            continue;
        }
        if (!active.empty()) {  // requests with no generations left (steps == 0) or a failed launch
            for (request_state* r : active)
                if (r->planned >= r->req.steps && !r->settled) {
                    const int rc = retire(r);
                    finish(r, rc, rc ? cb2_last_error() : "");
                }
            active.erase(std::remove_if(active.begin(), active.end(), [](request_state* r) { return r->settled; }),
                         active.end());
        }
    }
    sync_direct();
    cudaStreamSynchronize(stream);
    while (!inflight.empty()) {
        retire_round(inflight.front());
        inflight.pop_front();
    }
    for (request_state* r : active) finish(r, CB2_ETIMEOUT, "server stopped");
    active.clear();
    std::lock_guard<std::mutex> lock(mu);
    for (request_state* r : queue) {
        r->state = CB2_REQ_FAILED;
        r->error = CB2_ETIMEOUT;
        r->message = "server stopped";
        ++stats.failed;
    }
    queue.clear();
    cv_done.notify_all();
}

} // namespace cb2

using namespace cb2;

struct cb2_server {
    server_impl impl;
};

extern "C" {

int cb2_server_create(const cb2_server_opts* opts, cb2_server** out) {
    if (!out) return CB2_EINVAL;
    auto* s = new cb2_server();
    server_impl& m = s->impl;
    if (opts) m.opts = *opts;
    if (m.opts.chunk_steps <= 0) m.opts.chunk_steps = 128;
    if (m.opts.max_active <= 0) m.opts.max_active = 4096;
    // Defaults measured on the served mix (300 requests, sides up to 16384): chunks of
    // 8 generations and 128-row tiles 15.2 / 16.0 Tcell/s at 5000 / 20000 req/s with
    // p99 150 / 168 ms; 32 and 128 rows 17.0 / 17.7 (p99 134 / 151); 32 and 256 rows
    // 18.0 / 19.2 (p99 122 / 138).
    if (m.opts.temporal_steps <= 0) m.opts.temporal_steps = 32;
    const int k = m.opts.temporal_steps;
    if (k != 1 && k != 2 && k != 4 && k != 8 && k != 16 && k != 32) {
        delete s;
        set_error("server temporal_steps must be 1, 2, 4, 8, 16 or 32");
        return CB2_EINVAL;
    }
    const bool tile_rows_given = m.opts.tile_rows > 0;
    if (m.opts.tile_rows <= 0) m.opts.tile_rows = 256;
    if (m.opts.task_capacity <= 0) m.opts.task_capacity = 1 << 20;
    // Measured on the served mix (sides up to 16384): with 128-generation
    // rounds the batch kernel beats side-stream strip passes for every grid
    // of that mix, so only larger grids take them by default.
    if (m.opts.direct_cells == 0) m.opts.direct_cells = 1ll << 28;
    m.tiling.temporal_steps = m.opts.temporal_steps;
    m.tiling.tile_rows = m.opts.tile_rows;
    m.tiling.lowered_tile_rows = tile_rows_given ? m.opts.tile_rows : 64;
    m.t0 = clock_t_::now();
    cudaGetDevice(&m.device);
    size_t free_b = 0, total_b = 0;
    cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    if (m.opts.memory_budget == 0)
        m.opts.memory_budget = std::min<size_t>((size_t)150 << 30, free_b / 10 * 8);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking);
    for (int i = 0; i < kDirectStreams && e == cudaSuccess; ++i)
        e = cudaStreamCreateWithFlags(&m.direct[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m.ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = m.device;
        e = cudaMemPoolCreate(&m.pool, &props);
    }
    if (e == cudaSuccess) {
        uint64_t keep = UINT64_MAX;  // keep freed state in the pool for the next requests
        e = cudaMemPoolSetAttribute(m.pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) e = cudaMalloc(&m.d_sums, 17 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&m.h_sums, 17 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&m.d_slots, 16 * sizeof(unsigned long long) * (size_t)m.opts.max_active);
    if (e == cudaSuccess) e = cudaMallocHost(&m.h_slots, 16 * sizeof(unsigned long long) * (size_t)m.opts.max_active);
    for (int i = m.opts.max_active - 1; i >= 0; --i) m.free_slots.push_back(i);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("server setup: ") + cudaGetErrorString(e));
        if (m.stream) cudaStreamDestroy(m.stream);
        for (cudaStream_t d : m.direct)
            if (d) cudaStreamDestroy(d);
        if (m.ev_fork) cudaEventDestroy(m.ev_fork);
        if (m.pool) cudaMemPoolDestroy(m.pool);
        cudaFree(m.d_sums);
        cudaFreeHost(m.h_sums);
        delete s;
        return CB2_ECUDA;
    }
    // The batch engines' task arrays (device and pinned host) and their captured
    // launch graphs are set up here, before the first request, so that no
    // request waits for them (an engine set up by the first round added up to
    // ~0.2 s to every latency of a burst of arrivals).
    for (int i = 0; i < 2 && !m.opts.per_request; ++i) {
        int rc = m.engs[i].init(m.opts.task_capacity, m.opts.max_active, m.tiling.temporal_steps, m.opts.spin_limit);
        if (!rc) rc = m.engs[i].capture(kBatchBuiltin);
        if (!rc && generic_batch_kernel()) rc = m.engs[i].capture(kBatchAll);  // rounds holding lowered DSL rules
        if (rc) {
            for (int j = 0; j <= i; ++j) m.engs[j].release();
            for (cudaStream_t d : m.direct)
                if (d) cudaStreamDestroy(d);
            cudaEventDestroy(m.ev_fork);
            cudaStreamDestroy(m.stream);
            cudaMemPoolDestroy(m.pool);
            cudaFree(m.d_sums);
            cudaFreeHost(m.h_sums);
            cudaFree(m.d_slots);
            cudaFreeHost(m.h_slots);
            delete s;
            return rc;
        }
        m.engine_ready[i] = true;
    }
    m.thread = std::thread([&m] { m.loop(); });
    *out = s;
    return CB2_OK;
}

int cb2_server_submit(cb2_server* s, const cb2_request* req, int64_t* id) {
    if (!s || !req) {
        set_error("null server or request");
        return CB2_EINVAL;
    }
    server_impl& m = s->impl;
    grid_geom g;
    int rc = make_geom(req->automaton, req->x_size, req->y_size, &g);
    if (rc) return rc;
    if (req->steps < 0) {
        set_error("steps must be non-negative");
        return CB2_EINVAL;
    }
    const int max_thr = (int)(sizeof(req->thresholds) / sizeof(req->thresholds[0]));
    if (!req->host_cells && (req->n_thresholds < 0 || req->n_thresholds > max_thr ||
                             req->n_thresholds >= g.states)) {
        set_error("between 0 and (states - 1) thresholds are supported");
        return CB2_EINVAL;
    }
    auto r = std::make_unique<request_state>();
    r->req = *req;
    r->thr.assign(req->thresholds, req->thresholds + (req->host_cells ? 0 : req->n_thresholds));
    r->bytes = 2 * (size_t)g.planes * (size_t)g.plane_words * 4;
    if (r->bytes > m.opts.memory_budget) {
        set_error("request needs " + std::to_string(r->bytes) + " bytes of state, more than the server's budget of " +
                  std::to_string(m.opts.memory_budget));
        return CB2_ENOMEM;
    }
    std::lock_guard<std::mutex> lock(m.mu);
    r->id = m.next_id++;
    r->submit_s = m.now();
    if (id) *id = r->id;
    m.queue.push_back(r.get());
    m.reqs[r->id] = std::move(r);
    ++m.stats.submitted;
    m.cv_work.notify_one();
    return CB2_OK;
}

int cb2_server_status(cb2_server* s, int64_t id, cb2_request_status* st) {
    if (!s || !st) return CB2_EINVAL;
    server_impl& m = s->impl;
    std::lock_guard<std::mutex> lock(m.mu);
    auto it = m.reqs.find(id);
    if (it == m.reqs.end()) {
        set_error("unknown request " + std::to_string(id));
        return CB2_ENOTFOUND;
    }
    const request_state& r = *it->second;
    st->state = r.state;
    st->error = r.error;
    st->steps_done = r.done_steps;
    st->submit_s = r.submit_s;
    st->admit_s = r.admit_s;
    st->done_s = r.done_s;
    for (int i = 0; i < 16; ++i) st->checksum[i] = r.checksum[i];
    if (r.state == CB2_REQ_FAILED) set_error(r.message);
    return CB2_OK;
}

int cb2_server_wait(cb2_server* s, int64_t id, double timeout_s) {
    if (!s) return CB2_EINVAL;
    server_impl& m = s->impl;
    std::unique_lock<std::mutex> lock(m.mu);
    auto it = m.reqs.find(id);
    if (it == m.reqs.end()) {
        set_error("unknown request " + std::to_string(id));
        return CB2_ENOTFOUND;
    }
    request_state* r = it->second.get();
    const bool ok = m.cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), [&] {
        return r->state == CB2_REQ_DONE || r->state == CB2_REQ_FAILED;
    });
    if (!ok) {
        set_error("request " + std::to_string(id) + " not finished within the timeout");
        return CB2_ETIMEOUT;
    }
    if (r->state == CB2_REQ_FAILED) {
        set_error(r->message);
        return r->error;
    }
    return CB2_OK;
}

int cb2_server_drain(cb2_server* s, double timeout_s) {
    if (!s) return CB2_EINVAL;
    server_impl& m = s->impl;
    std::unique_lock<std::mutex> lock(m.mu);
    const bool ok = m.cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), [&] {
        return m.stats.completed + m.stats.failed >= m.stats.submitted;
    });
    if (!ok) {
        set_error("requests still pending after the timeout");
        return CB2_ETIMEOUT;
    }
    return CB2_OK;
}

int cb2_server_get_stats(cb2_server* s, cb2_server_stats* out) {
    if (!s || !out) return CB2_EINVAL;
    server_impl& m = s->impl;
    std::lock_guard<std::mutex> lock(m.mu);
    *out = m.stats;
    out->used_bytes = (int64_t)m.used_bytes;
    out->budget_bytes = (int64_t)m.opts.memory_budget;
    out->now_s = m.now();
    return CB2_OK;
}

int cb2_server_destroy(cb2_server* s) {
    if (!s) return CB2_OK;
    server_impl& m = s->impl;
    {
        std::lock_guard<std::mutex> lock(m.mu);
        m.stop = true;
        m.cv_work.notify_all();
    }
    if (m.thread.joinable()) m.thread.join();
    m.sync_direct();
    cudaStreamSynchronize(m.stream);
    for (int e = 0; e < 2; ++e)
        if (m.engine_ready[e]) m.engs[e].release();
    for (cudaEvent_t ev : m.spare_events) cudaEventDestroy(ev);
    cudaFree(m.d_sums);
    cudaFreeHost(m.h_sums);
    cudaFree(m.d_slots);
    cudaFreeHost(m.h_slots);
    cudaMemPoolDestroy(m.pool);
    cudaEventDestroy(m.ev_fork);
    for (cudaStream_t d : m.direct) cudaStreamDestroy(d);
    cudaStreamDestroy(m.stream);
    delete s;
    return CB2_OK;
}

} // extern "C"
