// cb2_dsl_configs.h -- the Cellato configs the library lowers (internal).
//
// CB2_DSL_CONFIGS(X) lists them in registry order, X(config, name): the
// bundled automata of the Cellato sources (src/automata/registry.hpp), the
// two user-defined examples of include/cellato_b200/dsl_examples.hpp, and the
// three automata that also have hand-written networks, again under
// "<name>:dsl".  A user's own automata follow, from the header named by
// CB2_USER_AUTOMATA that defines CB2_USER_CONFIGS(X) as a list of X(config)
// (registered under config::name).  cb2_generic.cu registers the list for
// the strip kernels and cb2_generic_batch.cu dispatches the batch kernel
// over it; both must see the same order, which this one list fixes.
#pragma once

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

#ifdef CB2_USER_AUTOMATA
#include CB2_USER_AUTOMATA
#endif

#define CB2_DSL_CONFIGS(X)                                                                                             \
    X(::brian::config, ::brian::config::name)                                                                          \
    X(::critters::config, ::critters::config::name)                                                                    \
    X(::cyclic::config, ::cyclic::config::name)                                                                        \
    X(::fire::config, ::fire::config::name)                                                                            \
    X(::fluid::config, ::fluid::config::name)                                                                          \
    X(::maze::config, ::maze::config::name)                                                                            \
    X(::traffic::config, ::traffic::config::name)                                                                      \
    X(::cellato_b200::examples::forest_fire_config, ::cellato_b200::examples::forest_fire_config::name)                \
    X(::cellato_b200::examples::noisy_life_config, ::cellato_b200::examples::noisy_life_config::name)                  \
    X(::game_of_life::config, "game-of-life:dsl")                                                                      \
    X(::wire::config, "wire:dsl")                                                                                      \
    X(::excitable::config, "excitable:dsl")
