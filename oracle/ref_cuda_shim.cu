// ref_cuda_shim.cu -- TEST AND MEASUREMENT INFRASTRUCTURE ONLY.
//
// A C-ABI driver around Cellato's OWN CUDA traversers, compiled straight from
// the reference headers by oracle/Makefile into
// oracle/_ref/libcellato_ref_cuda.so, so that the reference's GPU kernels can
// be timed on the same B200 as the kernels to beat and their results checked
// against this project's.  The product library never links or loads it.
//
//   traverser 0: cuda::simple   (traversers/cuda/simple.cuh:23-79), one
//                thread per word, one launch per generation
//   traverser 1: cuda::temporal (traversers/cuda/temporal.cuh:43-245), k
//                generations per launch in shared-memory tiles
//
// Automaton ids are oracle/ref_shim.cpp's (ref_automaton_id): the bundled
// set plus the two examples of include/cellato_b200/dsl_examples.hpp.
// Both traversers run over the reference's linear bit_planes layout with 64-bit words
// (memory/bit_planes_grid.hpp:35-271), the suites
// on_cuda::using_<uint64_t>::bit_planes / temporal_linear_bit_planes
// (experiments/test_suites.hpp:237-258).  Timing follows
// experiment_manager.hpp:132-154: CUDA events on the default stream around
// traverser.run(steps).
//
// The temporal kernel's (k, tile_y, block_y) are compile-time options
// (traversers/cuda/temporal_options.hpp:14-27, whose default set is the single
// point k=4, tile_y=32, block_y=8 and which documents editing the set).  This
// file supplies the option set below in place of that header, a superset of
// the default, so the sweep can search it.
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

#include "cellato/memory/idx_type.hpp"

#define CELLATO_CUDA_TEMPORAL_OPTIONS_HPP
namespace cellato::traversers::cuda::temporal::options {
using idx_type = cellato::memory::idx_type;
using block_size_x = std::integer_sequence<idx_type, 32>;
using time_steps = std::integer_sequence<idx_type, 2, 4, 8, 12, 16>;
using tile_size_y = std::integer_sequence<idx_type, 16, 32, 64>;
using block_size_y = std::integer_sequence<idx_type, 4, 8, 16>;
} // namespace cellato::traversers::cuda::temporal::options

#include "cellato/experiments/run_params.hpp"
#include "cellato/experiments/test_suites.hpp"
#include "cellato/traversers/cuda/simple.cuh"
#include "cellato/traversers/cuda/temporal.cuh"

#include "brian/config.hpp"
#include "critters/config.hpp"
#include "cyclic/config.hpp"
#include "excitable/config.hpp"
#include "fire/config.hpp"
#include "fluid/config.hpp"
#include "game_of_life/config.hpp"
#include "maze/config.hpp"
#include "traffic/config.hpp"
#include "wire/config.hpp"

#include "cellato_b200/dsl_examples.hpp"

namespace {

namespace ts = cellato::run::test_suites;

void put_error(char* err, int errlen, const std::string& msg) {
    if (err && errlen > 0) {
        std::strncpy(err, msg.c_str(), (std::size_t)errlen - 1);
        err[errlen - 1] = '\0';
    }
}

// One timed run of a suite on a grid whose planes the caller provides (P
// planes of y * x / 64 little-endian 64-bit words, concatenated).
template <typename suite>
int run_suite(int x, int y, int warm_steps, int steps, int k, int tile_y, int block_y, const void* planes_in,
              void* planes_out, float* ms_out) {
    using grid_t = typename suite::grid_t;
    using traverser_t = typename suite::traverser_t;
    using word_t = typename grid_t::store_type;

    grid_t grid((std::size_t)y, (std::size_t)x);
    auto planes = grid.data();
    const std::size_t words = grid.x_size_physical() * grid.y_size_physical();
    for (std::size_t p = 0; p < planes.size(); ++p)
        std::memcpy(planes[p], (const char*)planes_in + p * words * sizeof(word_t), words * sizeof(word_t));

    cellato::run::run_params params;
    params.x_size = x;
    params.y_size = y;
    params.steps = steps;
    params.word_size = 64;
    params.cuda_block_size_x = 32;
    params.cuda_block_size_y = block_y;
    params.temporal_steps = k;
    params.temporal_tile_size_y = tile_y;

    traverser_t traverser;
    traverser.init(grid, params);
    if (warm_steps > 0) traverser.run(warm_steps);
    CUCH(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    CUCH(cudaEventCreate(&e0));
    CUCH(cudaEventCreate(&e1));
    CUCH(cudaEventRecord(e0, 0));
    traverser.run(steps);
    CUCH(cudaEventRecord(e1, 0));
    CUCH(cudaEventSynchronize(e1));
    float ms = 0;
    CUCH(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CUCH(cudaGetLastError());
    if (ms_out) *ms_out = ms;

    grid_t result = traverser.fetch_result();
    if (planes_out) {
        auto out = result.data();
        for (std::size_t p = 0; p < out.size(); ++p)
            std::memcpy((char*)planes_out + p * words * sizeof(word_t), out[p], words * sizeof(word_t));
    }
    return 0;
}

template <typename automaton>
int with_traverser(int traverser, int x, int y, int warm_steps, int steps, int k, int tile_y, int block_y,
                   const void* in, void* out, float* ms) {
    switch (traverser) {
    case 0:
        return run_suite<ts::on_cuda::using_<std::uint64_t>::bit_planes<automaton>>(x, y, warm_steps, steps, k, tile_y,
                                                                                      block_y, in, out, ms);
    case 1:
        return run_suite<ts::on_cuda::using_<std::uint64_t>::temporal_linear_bit_planes<automaton>>(
            x, y, warm_steps, steps, k, tile_y, block_y, in, out, ms);
    default: return -2;
    }
}

} // namespace

extern "C" {

// Runs warm_steps untimed, then `steps` timed generations of the reference's
// CUDA traverser (0 simple, 1 temporal with k / tile_y / block_y) on the
// given planes; writes the final planes (after warm_steps + steps) and the
// timed milliseconds.  Returns 0, or a negative code with the message in err.
int ref_cuda_run(int automaton, int traverser, int x, int y, int warm_steps, int steps, int k, int tile_y,
                 int block_y, const void* planes_in, void* planes_out, float* ms, char* err, int errlen) {
    try {
        switch (automaton) {
        case 0:
            return with_traverser<game_of_life::config>(traverser, x, y, warm_steps, steps, k, tile_y, block_y,
                                                        planes_in, planes_out, ms);
        case 1:
            return with_traverser<wire::config>(traverser, x, y, warm_steps, steps, k, tile_y, block_y, planes_in,
                                                planes_out, ms);
        case 2:
            return with_traverser<excitable::config>(traverser, x, y, warm_steps, steps, k, tile_y, block_y,
                                                     planes_in, planes_out, ms);
#define CB2_REF_CASE(ID, CONFIG)                                                                                       \
    case ID:                                                                                                           \
        return with_traverser<CONFIG>(traverser, x, y, warm_steps, steps, k, tile_y, block_y, planes_in, planes_out, ms);
            CB2_REF_CASE(3, brian::config)
            CB2_REF_CASE(4, critters::config)
            CB2_REF_CASE(5, cyclic::config)
            CB2_REF_CASE(6, fire::config)
            CB2_REF_CASE(7, fluid::config)
            CB2_REF_CASE(8, maze::config)
            CB2_REF_CASE(9, traffic::config)
            CB2_REF_CASE(10, cellato_b200::examples::forest_fire_config)
            CB2_REF_CASE(11, cellato_b200::examples::noisy_life_config)
#undef CB2_REF_CASE
        default: put_error(err, errlen, "unknown automaton"); return -1;
        }
    } catch (const std::exception& e) {
        put_error(err, errlen, e.what());
        cudaGetLastError();
        return -3;
    }
}

} // extern "C"
