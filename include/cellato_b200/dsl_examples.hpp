// dsl_examples.hpp -- two user-defined automata written in the Cellato DSL
// (core/ast.hpp), the way a user adds a rule: a config with a name, an
// algorithm and a state dictionary.  The library lowers them like the
// bundled ones (cellato_b200/csrc/cb2_generic.cu) and registers them as
// "lightning-forest" and "noisy-life"; they are also the stochastic rules its
// tests check against the reference traverser, because no bundled automaton
// draws random numbers.
#pragma once

#include "cellato/core/ast.hpp"
#include "cellato/memory/state_dictionary.hpp"

namespace cellato_b200::examples {

using namespace cellato::ast;

// Drossel-Schwabl forest fire: a burning tree burns out; a tree catches fire
// from a burning neighbour or from lightning (probability 1/1000); an empty
// cell grows a tree with probability 3/100.  Both probabilities have
// recurring binary expansions, so the draws use the exact rational sampler.
enum class forest_cell { empty, tree, burning };

struct forest_fire {
    using empty = state_constant<forest_cell::empty>;
    using tree = state_constant<forest_cell::tree>;
    using burning = state_constant<forest_cell::burning>;

    using catches_fire =
        p<p<count_neighbors<burning, moore_8_neighbors>, greater_than, constant<0>>, or_, probability<1, 1000, 1>>;

    // clang-format off
    using algorithm =
        if_< p<current_state, equals, burning> >::then_<
            empty
        >::elif_< p<current_state, equals, tree> >::then_<
            if_< catches_fire >::then_< burning >::else_< tree >
        >::else_<
            if_< probability<3, 100, 2> >::then_< tree >::else_< empty >
        >;
    // clang-format on
};

struct forest_fire_config {
    static constexpr char name[] = "lightning-forest";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = forest_fire::algorithm;
    using cell_state = forest_cell;
    using state_dictionary =
        cellato::memory::grids::state_dictionary<forest_cell::empty, forest_cell::tree, forest_cell::burning>;
};

// Game of Life whose births happen with probability 3/4 (a dyadic ratio:
// two random words per draw) and whose survivors follow B3/S23 exactly.
enum class life_cell { dead, alive };

struct noisy_life {
    using dead = state_constant<life_cell::dead>;
    using alive = state_constant<life_cell::alive>;
    using n_alive = count_neighbors<alive, moore_8_neighbors>;

    // clang-format off
    using algorithm =
        if_< p<current_state, equals, alive> >::then_<
            if_< p<p<n_alive, equals, constant<2>>, or_, p<n_alive, equals, constant<3>>> >::then_< alive >::else_< dead >
        >::else_<
            if_< p<p<n_alive, equals, constant<3>>, and_, probability<3, 4, 5>> >::then_< alive >::else_< dead >
        >;
    // clang-format on
};

struct noisy_life_config {
    static constexpr char name[] = "noisy-life";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = noisy_life::algorithm;
    using cell_state = life_cell;
    using state_dictionary = cellato::memory::grids::state_dictionary<life_cell::dead, life_cell::alive>;
};

} // namespace cellato_b200::examples
