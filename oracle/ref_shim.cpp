// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A small C-ABI driver around Cellato's OWN CPU path, compiled straight from
// the reference headers by oracle/Makefile into oracle/_ref/libcellato_ref.so.
// It is the checker for the C restatement in cellato_oracle.c, the generator
// of the committed golden fixtures, and the CPU arm of the benchmark
// ("reference" kind).  The product library never links or loads it.
//
// It follows experiment_manager::run_round (experiments/experiment_manager.hpp:64-93):
// build a standard grid from the caller's cells, convert it to the suite's
// layout, init + run the CPU simple traverser (traversers/cpu/simple.hpp:19-95),
// fetch_result().to_standard(), and read get_checksum()
// (memory/standard_grid.hpp:182-218).  Cells cross the ABI as uint8 state
// dictionary indexes (memory/state_dictionary.hpp:10-42).

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "cellato/experiments/run_params.hpp"
#include "cellato/experiments/test_suites.hpp"

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

enum layout_id { L_STANDARD = 0, L_BIT_ARRAY = 1, L_BIT_PLANES = 2, L_TILED = 3 };

template <typename suite>
int run_suite(int x, int y, int steps, const uint8_t* in, uint8_t* out, char* checksum, int checksum_len,
              int seed = 42) {
    using automaton = typename suite::automaton;
    using dict = typename automaton::state_dictionary;
    using cell_t = typename suite::original_cell_t;
    using grid_t = typename suite::grid_t;
    using traverser_t = typename suite::traverser_t;

    cellato::run::run_params params;
    params.x_size = x;
    params.y_size = y;
    params.steps = steps;
    params.seed = seed;

    cellato::memory::grids::standard::grid<cell_t> initial(x, y);
    cell_t* data = initial.data();
    for (std::size_t i = 0; i < (std::size_t)x * (std::size_t)y; ++i) data[i] = dict::index_to_state(in[i]);

    grid_t grid = initial;
    traverser_t traverser;
    traverser.init(grid, params);
    traverser.run(steps);
    grid_t result = traverser.fetch_result();
    auto standard = result.to_standard();

    if (out) {
        const cell_t* res = standard.data();
        for (std::size_t i = 0; i < (std::size_t)x * (std::size_t)y; ++i) out[i] = (uint8_t)dict::state_to_index(res[i]);
    }
    if (checksum && checksum_len > 0) {
        std::string c = standard.get_checksum();
        std::strncpy(checksum, c.c_str(), (std::size_t)checksum_len - 1);
        checksum[checksum_len - 1] = '\0';
    }
    return 0;
}

template <typename automaton, typename fn_t>
int with_suite(int layout, int word_bits, fn_t&& fn) {
    switch (layout) {
    case L_STANDARD: return fn.template operator()<ts::on_cpu::standard<automaton>>();
    case L_BIT_ARRAY:
        if (word_bits == 32) return fn.template operator()<ts::on_cpu::using_<std::uint32_t>::bit_array<automaton>>();
        if (word_bits == 64) return fn.template operator()<ts::on_cpu::using_<std::uint64_t>::bit_array<automaton>>();
        return -3;
    case L_BIT_PLANES:
        if (word_bits == 32) return fn.template operator()<ts::on_cpu::using_<std::uint32_t>::bit_planes<automaton>>();
        if (word_bits == 64) return fn.template operator()<ts::on_cpu::using_<std::uint64_t>::bit_planes<automaton>>();
        return -3;
    case L_TILED:
        if (word_bits == 32)
            return fn.template operator()<ts::on_cpu::using_<std::uint32_t>::tiled_bit_planes<automaton>>();
        if (word_bits == 64)
            return fn.template operator()<ts::on_cpu::using_<std::uint64_t>::tiled_bit_planes<automaton>>();
        return -3;
    default: return -2;
    }
}

template <typename fn_t>
int with_automaton(int automaton, int layout, int word_bits, fn_t&& fn) {
    switch (automaton) {
    case 0: return with_suite<game_of_life::config>(layout, word_bits, fn);
    case 1: return with_suite<wire::config>(layout, word_bits, fn);
    case 2: return with_suite<excitable::config>(layout, word_bits, fn);
    case 3: return with_suite<brian::config>(layout, word_bits, fn);
    case 4: return with_suite<critters::config>(layout, word_bits, fn);
    case 5: return with_suite<cyclic::config>(layout, word_bits, fn);
    case 6: return with_suite<fire::config>(layout, word_bits, fn);
    case 7: return with_suite<fluid::config>(layout, word_bits, fn);
    case 8: return with_suite<maze::config>(layout, word_bits, fn);
    case 9: return with_suite<traffic::config>(layout, word_bits, fn);
    case 10: return with_suite<cellato_b200::examples::forest_fire_config>(layout, word_bits, fn);
    case 11: return with_suite<cellato_b200::examples::noisy_life_config>(layout, word_bits, fn);
    default: return -1;
    }
}

// The layout's host words, exactly as the reference grid stores them.
template <typename suite>
int pack_suite(int x, int y, const uint8_t* in, uint8_t* out, std::size_t out_len) {
    using automaton = typename suite::automaton;
    using dict = typename automaton::state_dictionary;
    using cell_t = typename suite::original_cell_t;
    using grid_t = typename suite::grid_t;

    cellato::memory::grids::standard::grid<cell_t> initial(x, y);
    cell_t* data = initial.data();
    for (std::size_t i = 0; i < (std::size_t)x * (std::size_t)y; ++i) data[i] = dict::index_to_state(in[i]);
    grid_t grid = initial;
    std::size_t written = 0;
    if constexpr (requires { grid.raw_data(); }) {
        using word_t = typename grid_t::store_type;
        std::size_t words = (std::size_t)x * (std::size_t)y / grid_t::cells_per_word;
        std::size_t bytes = words * sizeof(word_t);
        if (bytes > out_len) return -4;
        std::memcpy(out, grid.raw_data(), bytes);
        written = bytes;
    } else if constexpr (requires { grid.data().size(); }) {
        using word_t = typename grid_t::store_type;
        auto planes = grid.data();
        std::size_t words = grid.x_size_physical() * grid.y_size_physical();
        for (std::size_t p = 0; p < planes.size(); ++p) {
            if (written + words * sizeof(word_t) > out_len) return -4;
            std::memcpy(out + written, planes[p], words * sizeof(word_t));
            written += words * sizeof(word_t);
        }
    } else {
        return -2; // the standard layout has no packed words
    }
    return (int)written;
}

} // namespace

extern "C" {

// Runs `steps` generations of the reference CPU simple traverser with the
// requested layout (0 standard, 1 bit_array, 2 bit_planes, 3 tiled) and word
// size.  in/out hold x*y dictionary indexes; out and checksum may be null.
int ref_run(int automaton, int layout, int word_bits, int x, int y, int steps, const uint8_t* in, uint8_t* out,
            char* checksum, int checksum_len) {
    try {
        return with_automaton(automaton, layout, word_bits, [&]<typename suite>() {
            return run_suite<suite>(x, y, steps, in, out, checksum, checksum_len);
        });
    } catch (...) {
        return -10;
    }
}

// ref_run with the run's random seed (run_params::seed; 42 in ref_run).
int ref_run_seeded(int automaton, int layout, int word_bits, int x, int y, int steps, int seed, const uint8_t* in,
                   uint8_t* out, char* checksum, int checksum_len) {
    try {
        return with_automaton(automaton, layout, word_bits, [&]<typename suite>() {
            return run_suite<suite>(x, y, steps, in, out, checksum, checksum_len, seed);
        });
    } catch (...) {
        return -10;
    }
}

// The shim's automaton ids by the reference's names (config::name), -1 if unknown.
int ref_automaton_id(const char* name) {
    static const char* const names[] = {"game-of-life", "wire",  "excitable", "brian",   "critters",         "cyclic",
                                        "forest-fire",  "fluid", "maze",      "traffic", "lightning-forest", "noisy-life"};
    for (int i = 0; i < (int)(sizeof(names) / sizeof(names[0])); ++i)
        if (name && std::strcmp(name, names[i]) == 0) return i;
    return -1;
}

// Host byte image of the layout's grid words (bit_array, bit_planes, tiled).
int ref_pack(int automaton, int layout, int word_bits, int x, int y, const uint8_t* in, uint8_t* out, size_t out_len) {
    if (layout == L_STANDARD) return -2;
    try {
        return with_automaton(automaton, layout, word_bits, [&]<typename suite>() {
            return pack_suite<suite>(x, y, in, out, out_len);
        });
    } catch (...) {
        return -10;
    }
}

// Full-size runs: the reference CPU simple traverser with the bit_planes
// layout and 64-bit words over planes the caller provides (P planes of y rows
// of x/64 words, plane-major), skipping the standard grid, which at 65536^2
// would take 16 GiB of enum cells.  The grid is built with the reference's
// own sized constructor (memory/bit_planes_grid.hpp:71-78) and filled through
// data() (:202-212).  `planes` is overwritten with the result.  After
// generation checkpoints[i] (1 <= c <= steps) the planes are copied to
// snapshots[i] (same size as `planes`) from the traverser's per-step callback
// (traversers/cpu/simple.hpp:59-84).  Progress goes to stderr every
// `report_every` generations (0: never).  Returns 0, or a negative code.
int ref_run_planes64(int automaton, int x, int y, int steps, int seed, uint64_t* planes, const int* checkpoints,
                     int n_checkpoints, uint64_t* const* snapshots, int report_every) {
    try {
        return with_automaton(automaton, L_BIT_PLANES, 64, [&]<typename suite>() {
            using automaton_t = typename suite::automaton;
            if constexpr (!std::is_same_v<suite, ts::on_cpu::using_<std::uint64_t>::bit_planes<automaton_t>>) {
                return -3; // only the 64-bit bit_planes suite is requested (with_automaton is a runtime switch)
            } else {
            using grid_t = typename suite::grid_t;
            using traverser_t = typename suite::traverser_t;
            constexpr int P = grid_t::needed_bits;
            const std::size_t words = (std::size_t)y * (std::size_t)(x / 64);
            if (x % 64 || x <= 0 || y <= 0 || steps < 0) return -4;
            grid_t grid((std::size_t)y, (std::size_t)x);
            auto dst = grid.data();
            for (int p = 0; p < P; ++p) std::memcpy(dst[p], planes + p * words, words * sizeof(uint64_t));

            cellato::run::run_params params;
            params.x_size = x;
            params.y_size = y;
            params.steps = steps;
            params.seed = seed;
            traverser_t traverser;
            traverser.init(std::move(grid), params);
            auto t0 = std::chrono::steady_clock::now();
            traverser.run(steps, [&](int step, grid_t& g) {
                if (step <= 0) return;
                for (int i = 0; i < n_checkpoints; ++i)
                    if (checkpoints[i] == step) {
                        auto src = g.data();
                        for (int p = 0; p < P; ++p)
                            std::memcpy(snapshots[i] + p * words, src[p], words * sizeof(uint64_t));
                    }
                if (report_every > 0 && step % report_every == 0) {
                    double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                    std::fprintf(stderr, "ref_run_planes64: automaton %d generation %d/%d, %.1f s\n", automaton,
                                 step, steps, s);
                }
            });
            grid_t result = traverser.fetch_result();
            auto src = result.data();
            for (int p = 0; p < P; ++p) std::memcpy(planes + p * words, src[p], words * sizeof(uint64_t));
            return 0;
            }
        });
    } catch (...) {
        return -10;
    }
}

// Throughput sample of the reference CPU traverser (bit_planes layout, 64-bit
// words) on a grid given as planes (P planes of y rows of x/64 words): the
// rows are split into `threads` bands of y/threads rows, and each host thread
// runs the reference traverser on its band as a grid of its own (a torus of
// the band's rows), so the threads together advance every cell of the grid
// once per generation; threads = 1 runs the whole grid.  Returns the wall
// time in seconds of the slowest thread for `steps` generations (init and
// fetch outside the timed region), or a negative value on error.
double ref_bench_planes64(int automaton, int x, int y, int steps, int threads, const uint64_t* planes) {
    if (threads < 1 || x % 64 || x <= 0 || y % threads || steps < 0) return -2.0;
    const int rows = y / threads;
    std::vector<double> secs((std::size_t)threads, -1.0);
    std::atomic<int> ready{0};
    auto body = [&](int t) {
        int rc = -1;
        try {
            rc = with_automaton(automaton, L_BIT_PLANES, 64, [&]<typename suite>() {
                using automaton_t = typename suite::automaton;
                if constexpr (!std::is_same_v<suite, ts::on_cpu::using_<std::uint64_t>::bit_planes<automaton_t>>) {
                    return -3;
                } else {
                    using grid_t = typename suite::grid_t;
                    using traverser_t = typename suite::traverser_t;
                    constexpr int P = grid_t::needed_bits;
                    const std::size_t words = (std::size_t)y * (std::size_t)(x / 64);
                    const std::size_t band_words = (std::size_t)rows * (std::size_t)(x / 64);
                    grid_t grid((std::size_t)rows, (std::size_t)x);
                    auto dst = grid.data();
                    for (int p = 0; p < P; ++p)
                        std::memcpy(dst[p], planes + p * words + (std::size_t)t * band_words,
                                    band_words * sizeof(uint64_t));
                    cellato::run::run_params params;
                    params.x_size = x;
                    params.y_size = rows;
                    params.steps = steps;
                    traverser_t traverser;
                    traverser.init(std::move(grid), params);
                    ready.fetch_add(1);
                    while (ready.load() < threads) std::this_thread::yield();
                    auto t0 = std::chrono::steady_clock::now();
                    traverser.run(steps);
                    auto t1 = std::chrono::steady_clock::now();
                    secs[(std::size_t)t] = std::chrono::duration<double>(t1 - t0).count();
                    grid_t result = traverser.fetch_result();
                    (void)result;
                    return 0;
                }
            });
        } catch (...) {
        }
        if (rc != 0 && secs[(std::size_t)t] < 0) ready.fetch_add(1);  // release the others
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(body, t);
    for (auto& th : pool) th.join();
    double worst = 0;
    for (double s : secs) {
        if (s < 0) return -1.0;
        worst = s > worst ? s : worst;
    }
    return worst;
}

// Throughput sample for the CPU baseline: `threads` host threads each run an
// independent copy of the reference traverser on the same x*y input for
// `steps` generations.  Returns the wall time of the slowest thread in
// seconds (the traversers' init and fetch are outside the timed region), or
// a negative value on error.
double ref_bench(int automaton, int layout, int word_bits, int x, int y, int steps, int threads, const uint8_t* in) {
    if (threads < 1) threads = 1;
    std::vector<double> secs((std::size_t)threads, -1.0);
    std::atomic<int> ready{0};
    auto body = [&](int t) {
        try {
            with_automaton(automaton, layout, word_bits, [&]<typename suite>() {
                using automaton_t = typename suite::automaton;
                using dict = typename automaton_t::state_dictionary;
                using cell_t = typename suite::original_cell_t;
                using grid_t = typename suite::grid_t;
                using traverser_t = typename suite::traverser_t;
                cellato::run::run_params params;
                params.x_size = x;
                params.y_size = y;
                params.steps = steps;
                cellato::memory::grids::standard::grid<cell_t> initial(x, y);
                cell_t* data = initial.data();
                for (std::size_t i = 0; i < (std::size_t)x * (std::size_t)y; ++i)
                    data[i] = dict::index_to_state(in[i]);
                grid_t grid = initial;
                traverser_t traverser;
                traverser.init(grid, params);
                ready.fetch_add(1);
                while (ready.load() < threads) std::this_thread::yield();
                auto t0 = std::chrono::steady_clock::now();
                traverser.run(steps);
                auto t1 = std::chrono::steady_clock::now();
                secs[(std::size_t)t] = std::chrono::duration<double>(t1 - t0).count();
                grid_t result = traverser.fetch_result();
                (void)result;
                return 0;
            });
        } catch (...) {
            ready.fetch_add(1);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(body, t);
    for (auto& th : pool) th.join();
    double worst = 0;
    for (double s : secs) {
        if (s < 0) return -1.0;
        worst = s > worst ? s : worst;
    }
    return worst;
}

} // extern "C"
