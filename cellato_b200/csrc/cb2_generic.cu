// cb2_generic.cu -- the Cellato DSL automata lowered to strip kernels.
//
// Each automaton here is a Cellato config (name, algorithm, state
// dictionary): the bundled set of src/automata/registry.hpp, taken from the
// Cellato sources at build time; the two user-defined examples of
// include/cellato_b200/dsl_examples.hpp (stochastic rules); and the three
// automata that also have hand-written networks, registered again under
// "<name>:dsl" so the lowered path can be checked against those networks.  cb2_ast.cuh turns each
// config's algorithm into an ast_rule, and the strip kernels of
// cb2_launch.cuh run it: pipe_run_rows with a window of 3P words per row,
// one or two words per lane, a few levels per warp.
//
// A user's own automata join the table at build time: a header that defines
// their configs and the list macro CB2_USER_CONFIGS(X), e.g.
//     #define CB2_USER_CONFIGS(X) X(my_rules::config) X(other::config)
// named by `make USER_AUTOMATA=path/to/rules.hpp` (csrc/Makefile), is
// included here and each listed config is registered under its name.
//
// Built only when the Cellato headers are present (csrc/Makefile, CELLATO);
// cb2_generic_none.cpp stands in otherwise and registers nothing.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cb2_ast.cuh"
#include "cb2_dsl_configs.h"
#include "cellato_b200/fingerprint.hpp"
#include "cb2_internal.h"
#include "cb2_launch.cuh"

namespace cb2 {
namespace {

// The lowered plans of a DSL automaton: (K, V, L) with two rows per barrier.
// K = 1, 2 and 4 serve the remainders of a run; the window holds 3P words
// per row and level, so chains stay short.
template <class R>
const std::vector<strip_variant>& dsl_variants() {
    static const std::vector<strip_variant> v = {
        make_variant<R, 8, 1, 2, 2>(),  make_variant<R, 8, 1, 4, 2>(), make_variant<R, 1, 1, 1, 2>(),
        make_variant<R, 2, 1, 2, 2>(),  make_variant<R, 2, 1, 1, 2>(), make_variant<R, 4, 1, 2, 2>(),
        make_variant<R, 4, 1, 4, 2>(),  make_variant<R, 16, 1, 4, 2>(), make_variant<R, 16, 1, 2, 2>(),
        make_variant<R, 8, 2, 2, 2>(),  make_variant<R, 4, 1, 1, 2>(),
    };
    return v;
}

template <class Config>
struct dsl_entry {
    using dict = typename Config::state_dictionary;
    static const int64_t* values() {
        static int64_t v[dict::number_of_values];
        static bool done = false;
        if (!done) {
            for (int i = 0; i < dict::number_of_values; ++i) v[i] = (int64_t)dict::index_to_state(i);
            done = true;
        }
        return v;
    }
    static automaton_desc desc(const char* name) {
        constexpr uint64_t fp = ::cellato_b200::fingerprint::of<Config>();
        return automaton_desc{name, dict::needed_bits, dict::number_of_values, values(), fp};
    }
};

struct dsl_table {
    std::vector<automaton_desc> descs;
    std::vector<const std::vector<strip_variant>*> variants;
};

template <class Config>
void add(dsl_table& t, const char* name) {
    static_assert(Config::state_dictionary::needed_bits <= kMaxPlanes, "more bit-planes than the library supports");
    t.descs.push_back(dsl_entry<Config>::desc(name));
    t.variants.push_back(&dsl_variants<ast_rule<Config>>());
}

const dsl_table& table() {
    static const dsl_table t = [] {
        dsl_table d;
#define CB2_ADD_CONFIG(C, NAME) add<C>(d, NAME);
        CB2_DSL_CONFIGS(CB2_ADD_CONFIG)
#undef CB2_ADD_CONFIG
#ifdef CB2_USER_CONFIGS
#define CB2_ADD_USER_CONFIG(C) add<C>(d, C::name);
        CB2_USER_CONFIGS(CB2_ADD_USER_CONFIG)
#undef CB2_ADD_USER_CONFIG
#endif
        return d;
    }();
    return t;
}

} // namespace

uint64_t builtin_fingerprint(int id) {
    // the reference's own configs of the three automata the hand-written networks compute
    switch (id) {
    case 0: return ::cellato_b200::fingerprint::of<::game_of_life::config>();
    case 1: return ::cellato_b200::fingerprint::of<::wire::config>();
    case 2: return ::cellato_b200::fingerprint::of<::excitable::config>();
    default: return 0;
    }
}

int generic_count() { return (int)table().descs.size(); }

const automaton_desc* generic_desc(int i) {
    const dsl_table& t = table();
    return i >= 0 && i < (int)t.descs.size() ? &t.descs[(size_t)i] : nullptr;
}

const std::vector<strip_variant>& generic_variants(int i) {
    static const std::vector<strip_variant> none;
    const dsl_table& t = table();
    return i >= 0 && i < (int)t.variants.size() ? *t.variants[(size_t)i] : none;
}

} // namespace cb2
