// cellato_b200/traverser.hpp -- the B200 backend as a Cellato traverser.
//
// Header-only C++20 binding of the C-ABI (cellato_b200.h) to the reference's
// own types.  Include it from a Cellato build (it needs the reference headers
// on the include path) and link libcellato_b200.so.
//
//   cellato_b200::traverser<evaluator_t, grid_t, automaton>
//       the Traverser concept of traversers/cuda/simple.hpp:25-104:
//       is_CUDA, init(grid, run_params), run(steps[, callback]), fetch_result()
//       for the reference's standard, bit_array, bit_planes and
//       tiled_bit_planes grids (any word size the reference supports);
//   cellato_b200::b200_traverser_traits
//       the catalog traits of experiments/test_suites.hpp:127-173, so that
//       `--device CUDA --traverser b200` selects it;
//   cellato_b200::suites::using_<word>::bit_planes<automaton> (and friends)
//       suite types to list in suites_for (test_suites.hpp:259-285).
//
// The library holds precompiled rules looked up by the config's name; init()
// also compares the config's fingerprint (cellato_b200/fingerprint.hpp: its
// algorithm type and state dictionary) with the one the library registered
// under that name, so a config that reuses a registered name with another
// rule is rejected (std::invalid_argument) rather than run with the wrong one.
//
// Errors are rethrown with the reference's exception conventions
// (traversers/cuda_utils.cuh:37-47, traversers/cuda/temporal.hpp:57-83):
// CUDA failures as cellato_b200::cuda_error (a std::runtime_error),
// invalid configurations as std::invalid_argument, unknown automata as
// std::invalid_argument, cells outside the dictionary as std::out_of_range.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "cellato/experiments/run_params.hpp"
#include "cellato/experiments/test_suites.hpp"
#include "cellato/memory/bit_array_grid.hpp"
#include "cellato/memory/bit_planes_grid.hpp"
#include "cellato/memory/standard_grid.hpp"
#include "cellato/memory/tiled_bit_planes_grid.hpp"

#include "cellato_b200.h"
#include "cellato_b200/fingerprint.hpp"

namespace cellato_b200 {

class cuda_error : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

inline void check(int rc, const char* what) {
    if (rc >= 0) return;
    const std::string msg = std::string(what) + ": " + cb2_last_error();
    switch (rc) {
    case CB2_ECUDA: throw cuda_error(msg);
    case CB2_ESTATE: throw std::out_of_range(msg);
    case CB2_ENOMEM: throw std::runtime_error(msg);
    default: throw std::invalid_argument(msg);
    }
}

namespace detail {

namespace grids = cellato::memory::grids;

// How a reference grid type maps onto a C-ABI layout and host image.
template <typename grid_t, typename dict_t>
struct layout_of;

template <typename word_t, typename dict_t, grids::device dev>
struct layout_of<grids::bit_planes::grid<word_t, dict_t, dev>, dict_t> {
    using grid_t = grids::bit_planes::grid<word_t, dict_t, dev>;
    static constexpr int layout = CB2_LAYOUT_BIT_PLANES;
    static constexpr int word_bits = sizeof(word_t) * 8;
    static int64_t x(const grid_t& g) { return (int64_t)g.x_size_original(); }
    static int64_t y(const grid_t& g) { return (int64_t)g.y_size_original(); }
    static void save(const grid_t& g, std::vector<uint8_t>& img) {
        auto planes = g.data();
        const std::size_t bytes = g.x_size_physical() * g.y_size_physical() * sizeof(word_t);
        img.resize(bytes * planes.size());
        for (std::size_t p = 0; p < planes.size(); ++p) std::memcpy(img.data() + p * bytes, planes[p], bytes);
    }
    static grid_t load(int64_t x, int64_t y, const std::vector<uint8_t>& img) {
        grid_t g((std::size_t)y, (std::size_t)x);
        auto planes = g.data();
        const std::size_t bytes = g.x_size_physical() * g.y_size_physical() * sizeof(word_t);
        for (std::size_t p = 0; p < planes.size(); ++p) std::memcpy(planes[p], img.data() + p * bytes, bytes);
        return g;
    }
};

template <typename word_t, typename dict_t, grids::device dev>
struct layout_of<grids::tiled_bit_planes::grid<word_t, dict_t, dev>, dict_t> {
    using grid_t = grids::tiled_bit_planes::grid<word_t, dict_t, dev>;
    static constexpr int layout = CB2_LAYOUT_TILED_BIT_PLANES;
    static constexpr int word_bits = sizeof(word_t) * 8;
    static int64_t x(const grid_t& g) { return (int64_t)g.x_size_original(); }
    static int64_t y(const grid_t& g) { return (int64_t)g.y_size_original(); }
    static void save(const grid_t& g, std::vector<uint8_t>& img) {
        auto planes = g.data();
        const std::size_t bytes = g.x_size_physical() * g.y_size_physical() * sizeof(word_t);
        img.resize(bytes * planes.size());
        for (std::size_t p = 0; p < planes.size(); ++p) std::memcpy(img.data() + p * bytes, planes[p], bytes);
    }
    static grid_t load(int64_t x, int64_t y, const std::vector<uint8_t>& img) {
        grid_t g((std::size_t)y, (std::size_t)x);
        auto planes = g.data();
        const std::size_t bytes = g.x_size_physical() * g.y_size_physical() * sizeof(word_t);
        for (std::size_t p = 0; p < planes.size(); ++p) std::memcpy(planes[p], img.data() + p * bytes, bytes);
        return g;
    }
};

template <typename dict_t, typename word_t, grids::device dev>
struct layout_of<grids::bit_array::grid<dict_t, word_t, dev>, dict_t> {
    using grid_t = grids::bit_array::grid<dict_t, word_t, dev>;
    static constexpr int layout = CB2_LAYOUT_BIT_ARRAY;
    static constexpr int word_bits = sizeof(word_t) * 8;
    static int64_t x(const grid_t& g) { return (int64_t)g.x_size_logical(); }
    static int64_t y(const grid_t& g) { return (int64_t)g.y_size_logical(); }
    static std::size_t words(int64_t x, int64_t y) { return (std::size_t)(x * y) / grid_t::cells_per_word; }
    static void save(const grid_t& g, std::vector<uint8_t>& img) {
        const std::size_t bytes = words(x(g), y(g)) * sizeof(word_t);
        img.resize(bytes);
        std::memcpy(img.data(), g.raw_data(), bytes);
    }
    static grid_t load(int64_t x, int64_t y, const std::vector<uint8_t>& img) {
        grid_t g((std::size_t)y, (std::size_t)x);
        std::memcpy(g.raw_data(), img.data(), words(x, y) * sizeof(word_t));
        return g;
    }
};

// The standard layout carries enum values; the C-ABI takes dictionary indexes.
template <typename cell_t, typename dict_t, grids::device dev>
struct layout_of<grids::standard::grid<cell_t, dev>, dict_t> {
    using grid_t = grids::standard::grid<cell_t, dev>;
    static constexpr int layout = CB2_LAYOUT_STANDARD;
    static constexpr int word_bits = 8;
    static int64_t x(const grid_t& g) { return g.x_size_physical(); }
    static int64_t y(const grid_t& g) { return g.y_size_physical(); }
    static void save(const grid_t& g, std::vector<uint8_t>& img) {
        const std::size_t n = (std::size_t)x(g) * (std::size_t)y(g);
        img.resize(n);
        const cell_t* c = g.data();
        for (std::size_t i = 0; i < n; ++i) img[i] = (uint8_t)dict_t::state_to_index(c[i]);
    }
    static grid_t load(int64_t x, int64_t y, const std::vector<uint8_t>& img) {
        grid_t g((int)x, (int)y);
        cell_t* c = g.data();
        for (std::size_t i = 0; i < img.size(); ++i) c[i] = dict_t::index_to_state(img[i]);
        return g;
    }
};

struct grid_deleter {
    void operator()(cb2_grid* g) const { cb2_grid_destroy(g); }
};

} // namespace detail

// The Traverser concept over the C-ABI.  The grid is uploaded once by
// init(), advanced on the device by run(), and fetched (and freed) by
// fetch_result(), like the reference's CUDA traversers
// (traversers/cuda/simple.hpp:48-53, simple.cuh:81-89).
template <typename evaluator_type, typename grid_type, typename automaton>
class traverser {
    using grid_t = grid_type;
    using dict_t = typename automaton::state_dictionary;
    using layout = detail::layout_of<grid_t, dict_t>;

public:
    static constexpr bool is_CUDA = true;

    void init(grid_t grid, const cellato::run::run_params& params) {
        const int id = cb2_automaton_lookup(automaton::name);
        if (id < 0)
            throw std::invalid_argument(std::string("automaton '") + automaton::name +
                                        "' has no network in the B200 backend");
        uint64_t registered = 0;
        check(cb2_automaton_fingerprint(id, &registered), "cb2_automaton_fingerprint");
        constexpr uint64_t mine = fingerprint::of<automaton>();
        if (registered != mine) {
            char hex[64];
            std::snprintf(hex, sizeof hex, "%016llx, registered %016llx", (unsigned long long)mine,
                          (unsigned long long)registered);
            throw std::invalid_argument(std::string("automaton '") + automaton::name +
                                        "': this config's rule or state dictionary differs from the one the B200 "
                                        "library registered under that name (fingerprint " + hex +
                                        "); build the config into the library under a name of its own "
                                        "(make -C cellato_b200/csrc USER_AUTOMATA=...)");
        }
        _id = id;
        _x = layout::x(grid);
        _y = layout::y(grid);
        const int k = params.temporal_steps;
        _tuning = cb2_tuning{(k == 1 || k == 2 || k == 4 || k == 8 || k == 16 || k == 32) ? k : 0,
                             params.temporal_tile_size_y > 0 ? params.temporal_tile_size_y : 0, 0, 0, 0};
        cb2_grid* g = nullptr;
        check(cb2_grid_create(id, _x, _y, &g), "cb2_grid_create");
        _grid.reset(g);
        // stochastic rules draw with the run's seed (traversers/cpu/simple.hpp:30)
        check(cb2_grid_set_seed(_grid.get(), static_cast<uint64_t>(params.seed)), "cb2_grid_set_seed");
        std::vector<uint8_t> img;
        layout::save(grid, img);
        check(cb2_grid_upload(_grid.get(), layout::layout, layout::word_bits, img.data(), img.size(), nullptr),
              "cb2_grid_upload");
    }

    struct no_callback {};

    // Advances `steps` generations.  With a callback, it is called with
    // (generations done, host grid) before the first pass and after every
    // pass of the run's plan (temporal_steps generations, the last pass the
    // remainder), as the reference's temporal traverser calls back once per
    // chunk of temporal_steps (traversers/cuda/temporal.cuh:205-232).
    template <typename callback = no_callback>
    void run(int steps, callback&& callback_func = no_callback{}) {
        if (!_grid) throw std::logic_error("run() before init()");
        if constexpr (std::is_same_v<std::decay_t<callback>, no_callback>) {
            check(cb2_grid_run(_grid.get(), steps, &_tuning, nullptr), "cb2_grid_run");
        } else {
            cb2_tuning plan{};
            check(cb2_plan(_id, _x, _y, &_tuning, &plan), "cb2_plan");
            callback_func(0, current());
            for (int done = 0; done < steps;) {
                const int n = std::min(plan.temporal_steps, steps - done);
                check(cb2_grid_run(_grid.get(), n, &_tuning, nullptr), "cb2_grid_run");
                done += n;
                callback_func(done, current());
            }
        }
    }

    grid_t fetch_result() {
        grid_t out = current();
        _grid.reset();
        return out;
    }

private:
    grid_t current() const {
        const int64_t bytes = cb2_layout_bytes(_id, layout::layout, layout::word_bits, _x, _y);
        check((int)(bytes < 0 ? bytes : 0), "cb2_layout_bytes");
        std::vector<uint8_t> img((std::size_t)bytes);
        check(cb2_grid_download(_grid.get(), layout::layout, layout::word_bits, img.data(), img.size(), nullptr),
              "cb2_grid_download");
        return layout::load(_x, _y, img);
    }

    std::unique_ptr<cb2_grid, detail::grid_deleter> _grid;
    int _id = -1;
    int64_t _x = 0, _y = 0;
    cb2_tuning _tuning{0, 0, 0, 0};
};

// Catalog traits (experiments/test_suites.hpp:127-173): --device CUDA --traverser b200.
struct b200_traverser_traits {
    static constexpr const char* device_name = "CUDA";
    static constexpr const char* traverser_name = "b200";

    template <typename evaluator_t, typename grid_t, typename cellular_automaton>
    using type = traverser<evaluator_t, grid_t, cellular_automaton>;

    static bool options_match(const cellato::run::run_params&) { return true; }
};

// Suites to list in suites_for<automaton> (test_suites.hpp:259-285).
namespace suites {
namespace ts = cellato::run::test_suites::detail;

template <typename cellular_automaton>
using standard = ts::suite<cellular_automaton, ts::standard_layout, b200_traverser_traits>;

template <typename store_word_type>
struct using_ {
    template <typename cellular_automaton>
    using bit_array = ts::suite<cellular_automaton, ts::bit_array_layout<store_word_type>, b200_traverser_traits>;
    template <typename cellular_automaton>
    using bit_planes = ts::suite<cellular_automaton, ts::bit_planes_layout<store_word_type>, b200_traverser_traits>;
    template <typename cellular_automaton>
    using tiled_bit_planes =
        ts::suite<cellular_automaton, ts::tiled_bit_planes_layout<store_word_type>, b200_traverser_traits>;
};
} // namespace suites

} // namespace cellato_b200
