// Drop-in check: the B200 traverser registered as Cellato suites, driven by
// the reference's own experiment_manager::run_experiment(params, initial_state)
// (experiments/experiment_manager.hpp:43-57), must report the same checksum
// as the reference CPU simple traverser with the standard layout, for every
// layout and word size: game-of-life, wire and excitable (hand-written
// networks), every other bundled automaton and the two user-defined
// stochastic examples (lowered DSL).
// Exit status 0 = all equal, 1 = a mismatch, 77 = no CUDA device.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "cellato/experiments/experiment_manager.hpp"
#include "cellato/experiments/test_suites.hpp"
#include "cellato_b200/traverser.hpp"

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

namespace ts = cellato::run::test_suites;
namespace b2 = cellato_b200::suites;

static uint64_t mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <typename automaton>
std::vector<typename automaton::cell_state> initial(int x, int y, uint64_t seed) {
    using dict = typename automaton::state_dictionary;
    std::vector<typename automaton::cell_state> cells((std::size_t)x * y);
    for (std::size_t i = 0; i < cells.size(); ++i)
        cells[i] = dict::index_to_state((int)((mix(seed + (i + 1) * 0x9E3779B97F4A7C15ull) >> 11) % dict::number_of_values));
    return cells;
}

static int failures = 0;

template <typename suite, typename automaton>
std::string checksum(const cellato::run::run_params& p, const std::vector<typename automaton::cell_state>& init) {
    cellato::run::experiment_manager<suite> m;
    return m.run_experiment(p, init).checksums.at(0);
}

template <typename automaton, typename b200_suite>
void compare(const char* label, int x, int y, int steps, int temporal_steps, int seed = 42) {
    cellato::run::run_params p;
    p.automaton = automaton::name;
    p.x_size = x;
    p.y_size = y;
    p.steps = steps;
    p.temporal_steps = temporal_steps;
    p.seed = seed;
    const auto init = initial<automaton>(x, y, 7 + steps);
    const std::string want = checksum<ts::on_cpu::standard<automaton>, automaton>(p, init);
    const std::string got = checksum<b200_suite, automaton>(p, init);
    const bool ok = want == got;
    failures += !ok;
    std::printf("%-10s %-26s %5dx%-4d %3d steps  %s\n", automaton::name, label, x, y, steps, ok ? "ok" : "MISMATCH");
    if (!ok) std::printf("  reference %s\n  b200      %s\n", want.c_str(), got.c_str());
}

template <typename A>
void all_layouts(int x, int y, int steps, int seed = 42) {
    compare<A, b2::standard<A>>("standard", x, y, steps, 0, seed);
    compare<A, b2::using_<uint32_t>::bit_planes<A>>("bit_planes u32 k8", x, y, steps, 8, seed);
    compare<A, b2::using_<uint64_t>::bit_planes<A>>("bit_planes u64", x, y, steps, 0, seed);
    compare<A, b2::using_<uint32_t>::bit_array<A>>("bit_array u32 k4", x, y, steps, 4, seed);
    compare<A, b2::using_<uint64_t>::bit_array<A>>("bit_array u64", x, y, steps, 0, seed);
    compare<A, b2::using_<uint32_t>::tiled_bit_planes<A>>("tiled u32 k16", x, y, steps, 16, seed);
    compare<A, b2::using_<uint64_t>::tiled_bit_planes<A>>("tiled u64", x, y, steps, 0, seed);
}

int main() {
    try {
        // 6720 is divisible by every word's cells_per_word (32, 64, 16, 10, 21).
        all_layouts<game_of_life::config>(6720, 16, 9);
        all_layouts<wire::config>(6720, 24, 13);
        all_layouts<excitable::config>(6720, 16, 21);
        // lowered DSL automata (6720 is also divisible by 6, 8, 12 and 16 cells per word)
        all_layouts<brian::config>(6720, 16, 11);
        all_layouts<critters::config>(6720, 24, 10);
        all_layouts<cyclic::config>(6720, 16, 9);
        all_layouts<fire::config>(6720, 16, 12);
        all_layouts<fluid::config>(6720, 16, 15);
        all_layouts<maze::config>(6720, 16, 8);
        all_layouts<traffic::config>(6720, 24, 14);
        all_layouts<cellato_b200::examples::forest_fire_config>(6720, 16, 17, 9);
        all_layouts<cellato_b200::examples::noisy_life_config>(6720, 16, 13, 1234);
        // the traverser also reports through the suite catalog
        cellato::run::run_params p;
        p.automaton = "wire";
        p.device = "CUDA";
        p.traverser = "b200";
        p.evaluator = p.layout = "bit_planes";
        p.word_size = 64;
        if (!b2::using_<uint64_t>::bit_planes<wire::config>::is_for(p)) {
            std::printf("suite::is_for did not select the b200 suite\n");
            ++failures;
        }
    } catch (const cellato_b200::cuda_error& e) {
        std::printf("no usable CUDA device: %s\n", e.what());
        return 77;
    }
    std::printf("%s\n", failures ? "FAILED" : "all equal");
    return failures ? 1 : 0;
}
