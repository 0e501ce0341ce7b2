// Fingerprint check: the drop-in traverser binds a config to the library's
// rule by type, not by name.  Needs no GPU (the check happens in init()
// before any device call).
//   1. every bundled config's fingerprint, computed here from the reference
//      headers, equals the one the library registered under its name;
//   2. distinct rules have distinct fingerprints;
//   3. a config named "game-of-life" whose rule is HighLife (B36/S23), and
//      one named "wire" with a reordered state dictionary, are rejected by
//      traverser::init with std::invalid_argument.
// Exit status 0 = all as expected, 1 = a failure.
#include <cstdint>
#include <cstdio>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "cellato/core/ast.hpp"
#include "cellato/experiments/run_params.hpp"
#include "cellato/memory/standard_grid.hpp"
#include "cellato/memory/state_dictionary.hpp"
#include "cellato_b200/fingerprint.hpp"
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

namespace highlife {
using namespace cellato::ast;
using game_of_life::gol_cell_state;
using alive = state_constant<gol_cell_state::alive>;
using dead = state_constant<gol_cell_state::dead>;
using count = count_neighbors<alive, moore_8_neighbors>;
using survives = p<p<count, equals, constant<2>>, or_, p<count, equals, constant<3>>>;
using born = p<p<count, equals, constant<3>>, or_, p<count, equals, constant<6>>>;
// clang-format off
using algorithm =
    if_< p<current_state, equals, alive> >::then_<
        if_< survives >::then_< alive >::else_< dead >
    >::else_<
        if_< born >::then_< alive >::else_< dead >
    >;
// clang-format on

// HighLife under Game of Life's name and dictionary.
struct config {
    static constexpr char name[] = "game-of-life";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = highlife::algorithm;
    using cell_state = gol_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell_state::dead, cell_state::alive>;
};
} // namespace highlife

// WireWorld's rule under its name, with the dictionary's order changed.
struct wire_reordered {
    static constexpr char name[] = "wire";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = wire::config::algorithm;
    using cell_state = wire::config::cell_state;
    using state_dictionary =
        cellato::memory::grids::state_dictionary<cell_state::empty, cell_state::conductor, cell_state::electron_head,
                                                 cell_state::electron_tail>;
};

static int failures = 0;
static std::set<uint64_t> seen;

template <typename C>
void registered(const char* name) {
    constexpr uint64_t mine = cellato_b200::fingerprint::of<C>();
    const int id = cb2_automaton_lookup(name);
    uint64_t lib = 0;
    const int rc = id < 0 ? id : cb2_automaton_fingerprint(id, &lib);
    const bool ok = rc == CB2_OK && lib == mine;
    failures += !ok;
    std::printf("%-20s %016llx  %s\n", name, (unsigned long long)mine, ok ? "ok" : "MISMATCH");
    if (!ok) std::printf("  library: rc %d, %016llx (%s)\n", rc, (unsigned long long)lib, cb2_last_error());
    if (std::string(name).find(":dsl") == std::string::npos && !seen.insert(mine).second) {
        std::printf("  fingerprint %016llx seen twice\n", (unsigned long long)mine);
        ++failures;
    }
}

template <typename C>
void rejected(const char* label) {
    using dict = typename C::state_dictionary;
    using grid_t = cellato::memory::grids::standard::grid<typename C::cell_state>;
    cellato_b200::traverser<void, grid_t, C> t;
    cellato::run::run_params p;
    p.x_size = 64;
    p.y_size = 8;
    grid_t g(64, 8);
    for (std::size_t i = 0; i < 64 * 8; ++i) g.data()[i] = dict::index_to_state(0);
    bool ok = false;
    try {
        t.init(g, p);
    } catch (const std::invalid_argument& e) {
        ok = std::string(e.what()).find("differs") != std::string::npos;
        std::printf("%-20s rejected: %s\n", label, e.what());
    } catch (const std::exception& e) {
        std::printf("%-20s wrong exception: %s\n", label, e.what());
    }
    if (!ok) std::printf("%-20s NOT REJECTED\n", label);
    failures += !ok;
}

int main() {
    registered<game_of_life::config>("game-of-life");
    registered<wire::config>("wire");
    registered<excitable::config>("excitable");
    registered<game_of_life::config>("game-of-life:dsl");
    registered<wire::config>("wire:dsl");
    registered<excitable::config>("excitable:dsl");
    registered<brian::config>("brian");
    registered<critters::config>("critters");
    registered<cyclic::config>("cyclic");
    registered<fire::config>("forest-fire");
    registered<fluid::config>("fluid");
    registered<maze::config>("maze");
    registered<traffic::config>("traffic");
    registered<cellato_b200::examples::forest_fire_config>("lightning-forest");
    registered<cellato_b200::examples::noisy_life_config>("noisy-life");
    if (cellato_b200::fingerprint::of<highlife::config>() == cellato_b200::fingerprint::of<game_of_life::config>()) {
        std::printf("HighLife and Game of Life share a fingerprint\n");
        ++failures;
    }
    rejected<highlife::config>("highlife as gol");
    rejected<wire_reordered>("wire reordered");
    std::printf("%s\n", failures ? "FAILED" : "fingerprints ok");
    return failures ? 1 : 0;
}
