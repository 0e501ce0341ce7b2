// cb2_band.cpp -- entry points for a grid split into row bands across GPUs.
//
// Each rank holds its band of rows plus `ghost` rows above and below in
// caller-owned planes (rows_total = band + 2 * ghost).  Before a pass of K
// generations (K <= ghost), the K ghost rows next to the band are refreshed
// from the neighbouring ranks (a halo exchange the caller runs, e.g. NCCL
// send/recv of contiguous rows); the pass then writes only the band's rows,
// reading the ghosts for the rows it needs outside the band.  The seeded
// input and the checksum are defined on the global grid, so a band run gives
// the same cells and the same 16 tile sums as one grid of the global size.
#include "cellato_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "cb2_internal.h"

namespace cb2 {
namespace {

int check_planes(const grid_geom& g, const void* const* planes, const char* what) {
    if (!planes) {
        set_error(std::string("null ") + what + " plane array");
        return CB2_EINVAL;
    }
    for (int p = 1; p < g.planes; ++p)
        if ((const char*)planes[p] - (const char*)planes[0] != (ptrdiff_t)(p * g.plane_words * 4)) {
            set_error(std::string(what) + " planes must be consecutive in one allocation (stride = rows * x_size / 8 bytes)");
            return CB2_EINVAL;
        }
    return CB2_OK;
}

int cuda_err(cudaError_t e, const char* what) {
    cudaGetLastError();
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CB2_ECUDA;
}

} // namespace
} // namespace cb2

using namespace cb2;

extern "C" {

int cb2_band_pass(int automaton, void* const* in, void* const* out, int64_t x_size, int64_t rows_total,
                  int64_t row_first, int64_t rows_out, int temporal_steps, const cb2_tuning* tuning, void* stream) {
    if (automaton >= kNumBuiltin && automaton < automaton_count()) {
        // A lowered DSL rule may read the cells' generation and global row
        // (Margolus blocks, probability draws), which only cb2_band_pass_at knows.
        set_error("a lowered DSL automaton needs the band's global rows and generation: use cb2_band_pass_at");
        return CB2_EINVAL;
    }
    return cb2_band_pass_at(automaton, in, out, x_size, rows_total, row_first, rows_out, temporal_steps, 0,
                            kDefaultSeed, 0, rows_total, tuning, stream);
}

int cb2_band_pass_at(int automaton, void* const* in, void* const* out, int64_t x_size, int64_t rows_total,
                     int64_t row_first, int64_t rows_out, int temporal_steps, int64_t time_step, uint64_t seed,
                     int64_t global_row0, int64_t global_rows, const cb2_tuning* tuning, void* stream) {
    grid_geom g;
    int rc = make_geom(automaton, x_size, rows_total, &g);
    if (rc) return rc;
    if (time_step < 0 || global_rows < 1) {
        set_error("negative time_step or empty global grid");
        return CB2_EINVAL;
    }
    if ((rc = check_planes(g, in, "input")) || (rc = check_planes(g, out, "output"))) return rc;
    if (row_first < 0 || rows_out < 1 || row_first + rows_out > rows_total) {
        set_error("band rows outside the planes");
        return CB2_EINVAL;
    }
    if (row_first < temporal_steps || rows_total - (row_first + rows_out) < temporal_steps) {
        set_error("a pass of " + std::to_string(temporal_steps) + " generations needs that many ghost rows each side");
        return CB2_EINVAL;
    }
    cb2_tuning t{temporal_steps, 0, 0, 0, 0};
    if (tuning) {
        t = *tuning;
        t.temporal_steps = temporal_steps;
    }
    grid_geom window = g;  // plan the tiles for the band's rows
    window.h = (int32_t)rows_out;
    window.y_size = rows_out;
    window.plane_words = (int64_t)g.wd * rows_out;
    run_plan plan;
    rc = resolve_plan(window, &t, &plan);
    if (rc) return rc;
    int64_t row0 = global_row0 % global_rows;  // the planes' row 0 (a ghost row for rank 0) as a global row
    if (row0 < 0) row0 += global_rows;
    cudaError_t e = launch_strip_window(g, (const uint32_t*)in[0], (uint32_t*)out[0], plan, (int)row_first,
                                        (int)rows_out, (cudaStream_t)stream, time_step, seed, row0, global_rows);
    if (e != cudaSuccess) return cuda_err(e, "band pass launch");
    return CB2_OK;
}

int64_t cb2_band_schedule(int64_t steps, int temporal_steps, int ghost, int* depths, int64_t capacity) {
    if (steps < 0 || temporal_steps < 1 || ghost < 1 || capacity < 0 || (capacity && !depths)) {
        set_error("band schedule needs steps >= 0, temporal_steps >= 1, ghost >= 1 and room for the depths");
        return CB2_EINVAL;
    }
    const int k_main = temporal_steps < ghost ? temporal_steps : ghost;
    int64_t n = 0, left = steps;
    while (left > 0) {
        int k = k_main;
        while (k > left) k /= 2;  // the remainder's binary digits, largest first
        if (n < capacity) depths[n] = k;
        ++n;
        left -= k;
    }
    return n;
}

int cb2_band_run(int automaton, void* const* a, void* const* b, int64_t x_size, int64_t band_rows, int ghost,
                 int64_t time_step, int64_t steps, uint64_t seed, int64_t global_row0, int64_t global_rows,
                 const cb2_tuning* tuning, cb2_halo_exchange_fn exchange, void* user, void* stream,
                 void* exchange_stream, int* result_in_b) {
    if (!exchange || band_rows < 1 || ghost < 1 || steps < 0 || time_step < 0) {
        set_error("band run needs an exchange function, band rows, ghost rows, steps >= 0 and time_step >= 0");
        return CB2_EINVAL;
    }
    const int64_t rows_total = band_rows + 2 * (int64_t)ghost;
    grid_geom g;
    int rc = make_geom(automaton, x_size, rows_total, &g);
    if (rc) return rc;
    if ((rc = check_planes(g, a, "a")) || (rc = check_planes(g, b, "b"))) return rc;
    int k_main = tuning && tuning->temporal_steps ? tuning->temporal_steps : 0;
    if (!k_main) {  // the single-grid plan of a grid of the band's size
        grid_geom band = g;
        band.h = (int32_t)band_rows;
        band.y_size = band_rows;
        band.plane_words = (int64_t)g.wd * band_rows;
        cb2_tuning t0{0, 0, 0, 0, 0};
        run_plan p;
        if ((rc = resolve_plan(band, &t0, &p))) return rc;
        k_main = p.k;
    }
    if (band_rows < std::min(k_main, ghost)) {
        // the exchange copies the neighbours' first / last k band rows
        set_error("bands of " + std::to_string(band_rows) + " rows are thinner than a pass of " +
                  std::to_string(std::min(k_main, ghost)) + " generations");
        return CB2_EINVAL;
    }
    const int64_t n = cb2_band_schedule(steps, k_main, ghost, nullptr, 0);
    if (n < 0) return (int)n;
    std::vector<int> depths((size_t)n);
    cb2_band_schedule(steps, k_main, ghost, depths.data(), n);

    cudaStream_t s = (cudaStream_t)stream, xs = (cudaStream_t)exchange_stream;
    cudaEvent_t ready = nullptr, landed = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&landed, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (ready) cudaEventDestroy(ready);
        return cuda_err(e, "band run events");
    }
    void* const* bufs[2] = {a, b};
    int cur = 0;
    int64_t t = time_step;
    const int64_t planes_row0 = global_row0 - ghost;  // global row of the planes' row 0
    for (int k : depths) {
        // The exchange may only overwrite ghost rows once the previous pass,
        // which read them, is done; it reads band rows that pass wrote.
        if ((e = cudaEventRecord(ready, s)) != cudaSuccess || (e = cudaStreamWaitEvent(xs, ready, 0)) != cudaSuccess)
            break;
        if ((rc = exchange(user, cur, k, exchange_stream)) != 0) {
            set_error("halo exchange callback failed with " + std::to_string(rc));
            rc = CB2_EINVAL;
            break;
        }
        const bool split = band_rows >= 3 * (int64_t)k;
        if (split && (rc = cb2_band_pass_at(automaton, bufs[cur], bufs[1 - cur], x_size, rows_total, ghost + k,
                                            band_rows - 2 * k, k, t, seed, planes_row0, global_rows, tuning,
                                            stream)))
            break;
        if ((e = cudaEventRecord(landed, xs)) != cudaSuccess || (e = cudaStreamWaitEvent(s, landed, 0)) != cudaSuccess)
            break;
        if (split) {
            if ((rc = cb2_band_pass_at(automaton, bufs[cur], bufs[1 - cur], x_size, rows_total, ghost, k, k, t, seed,
                                       planes_row0, global_rows, tuning, stream)) ||
                (rc = cb2_band_pass_at(automaton, bufs[cur], bufs[1 - cur], x_size, rows_total,
                                       ghost + band_rows - k, k, k, t, seed, planes_row0, global_rows, tuning,
                                       stream)))
                break;
        } else if ((rc = cb2_band_pass_at(automaton, bufs[cur], bufs[1 - cur], x_size, rows_total, ghost, band_rows,
                                          k, t, seed, planes_row0, global_rows, tuning, stream))) {
            break;
        }
        cur ^= 1;
        t += k;
    }
    cudaEventDestroy(ready);
    cudaEventDestroy(landed);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_err(e, "band run stream ordering");
    if (result_in_b) *result_in_b = cur;
    return CB2_OK;
}

int cb2_fill_random_planes(int automaton, void* const* planes, int64_t x_size, int64_t rows, int64_t global_row0,
                           int64_t global_rows, uint64_t seed, const uint64_t* thresholds, int n_thresholds,
                           void* stream) {
    grid_geom g;
    int rc = make_geom(automaton, x_size, rows, &g);
    if (rc) return rc;
    if ((rc = check_planes(g, planes, "output"))) return rc;
    if (global_rows < 1 || n_thresholds < 0 || n_thresholds > kMaxThresholds || n_thresholds >= g.states ||
        (n_thresholds && !thresholds)) {
        set_error("invalid global rows or thresholds");
        return CB2_EINVAL;
    }
    cudaError_t e = launch_fill_random_rows(g, (uint32_t*)planes[0], seed, thresholds, n_thresholds, global_row0,
                                            global_rows, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_err(e, "fill launch");
    return CB2_OK;
}

int cb2_checksum_planes(int automaton, const void* const* planes, int64_t x_size, int64_t rows, int64_t row_first,
                        int64_t row_count, int64_t global_row0, int64_t global_rows, const int64_t* values,
                        int n_values, uint64_t out[16], void* stream) {
    grid_geom g;
    int rc = make_geom(automaton, x_size, rows, &g);
    if (rc) return rc;
    if ((rc = check_planes(g, planes, "input"))) return rc;
    if (!out || n_values < 0 || n_values > (1 << kMaxPlanes) || (n_values && !values)) {
        set_error("null output or more than " + std::to_string(1 << kMaxPlanes) + " state values");
        return CB2_EINVAL;
    }
    if (!values) {  // the dictionary's own state values, as the reference's standard grid sums them
        values = automaton_at(automaton)->values;
        n_values = automaton_at(automaton)->states;
    }
    if (row_first < 0 || row_count < 0 || row_first + row_count > rows || global_row0 < 0 ||
        global_row0 + row_count > global_rows) {
        set_error("checksum rows outside the planes or the global grid");
        return CB2_EINVAL;
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long* sums = nullptr;
    cudaError_t e = cudaMallocAsync(&sums, 16 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(sums, 0, 16 * sizeof(unsigned long long), s);
    if (e == cudaSuccess)
        e = launch_checksum_rows(g, (const uint32_t*)planes[0], values, n_values, row_first, row_count, global_row0,
                                 global_rows, sums, s);
    unsigned long long host[16] = {};
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, sums, sizeof(host), cudaMemcpyDeviceToHost, s);
    if (sums) cudaFreeAsync(sums, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err(e, "band checksum");
    for (int i = 0; i < 16; ++i) out[i] = host[i];
    return CB2_OK;
}

} // extern "C"
