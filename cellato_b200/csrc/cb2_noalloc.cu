// cb2_noalloc.cu -- cb2_run_bit_planes_in_place: advancing a grid without any
// device allocation.
//
// Some callers cannot call cudaMalloc: a host application that owns all
// device memory through its own pool and forbids plugins to allocate, or a
// loop that must not risk the implicit synchronisation and failure modes of a
// fresh allocation between steps.  They can hand over only the grid itself.
// The strip kernels need a second buffer to write the next generation into;
// here that buffer is a file-scope __device__ array of a fixed size, which
// every GPU that loads this library holds until the process exits.
//
// Host code must not use g_scratch's name as a device address: on the host
// it is only a stand-in for the symbol.  The device address is looked up
// once per device with cudaGetSymbolAddress (on the first call made while
// that device is current) and passed to the kernels like any other buffer.
#include "cellato_b200.h"

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>

#include "cb2_internal.h"

namespace {

constexpr size_t kScratchBytes = CB2_STATIC_SCRATCH_BYTES;

// The second buffer of the in-place run.  Shared by every call on a device
// and never cleared: each launch writes every word of the generation it
// produces before anything reads it.
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
std::map<int, void*> g_scratch_addr;  // device ordinal -> device address of g_scratch

int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cb2::set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return CB2_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_scratch_addr.find(dev);
    if (it != g_scratch_addr.end()) {
        *out = it->second;
        return CB2_OK;
    }
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess || !ptr) {
        cb2::set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        return CB2_ECUDA;
    }
    g_scratch_addr[dev] = ptr;
    *out = ptr;
    return CB2_OK;
}

} // namespace

extern "C" int cb2_run_bit_planes_in_place(int automaton, void* const* planes, int64_t x_size, int64_t y_size,
                                           int64_t time_step, int64_t steps, uint64_t seed, const cb2_tuning* tuning,
                                           void* stream) {
    cb2::grid_geom g;
    int rc = cb2::make_geom(automaton, x_size, y_size, &g);
    if (rc) return rc;
    if (!planes || steps < 0 || time_step < 0) {
        cb2::set_error("null plane array, negative steps or negative time_step");
        return CB2_EINVAL;
    }
    const size_t bytes = (size_t)g.planes * (size_t)g.plane_words * 4;
    if (bytes > kScratchBytes) {
        cb2::set_error("grid of " + std::to_string(bytes) + " bytes of bit-planes exceeds the " +
                       std::to_string(kScratchBytes) + "-byte static scratch of cb2_run_bit_planes_in_place; "
                       "use cb2_run_bit_planes with a caller-owned second buffer");
        return CB2_EINVAL;
    }
    for (int p = 1; p < g.planes; ++p)
        if ((char*)planes[p] - (char*)planes[0] != (ptrdiff_t)(p * g.plane_words * 4)) {
            cb2::set_error("planes must be consecutive in one allocation (stride = y_size * x_size / 8 bytes)");
            return CB2_EINVAL;
        }
    void* scratch = nullptr;
    rc = scratch_address(&scratch);
    if (rc) return rc;
    uint32_t* const bufs[2] = {(uint32_t*)planes[0], (uint32_t*)scratch};
    int res = 0;
    rc = cb2::run_chunks(g, bufs, 0, steps, tuning, (cudaStream_t)stream, &res, time_step, seed);
    if (rc) return rc;
    if (res == 1) {  // an odd number of passes left the result in the scratch
        cudaError_t e = cudaMemcpyAsync(planes[0], scratch, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
        if (e != cudaSuccess) {
            cb2::set_error(std::string("copy back from scratch: ") + cudaGetErrorString(e));
            return CB2_ECUDA;
        }
    }
    return CB2_OK;
}
