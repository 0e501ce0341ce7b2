// cellato_b200/fingerprint.hpp -- a compile-time fingerprint of a Cellato
// automaton's rule and state dictionary.
//
// The reference picks an automaton's code by its type: a suite is
// instantiated for the config and always evaluates that config's own
// algorithm (experiments/test_suites.hpp:189-195).  The B200 library holds
// precompiled rules and is looked up by name, so the drop-in traverser checks
// that the rule registered under a name is the rule the caller's config
// spells: both sides hash the config's algorithm type structurally (each AST
// node of core/ast.hpp:15-151 as a tag, its integer parameters and its
// children, depth first) together with its state dictionary (number of
// states, bit-planes, each state's value in index order,
// memory/state_dictionary.hpp:10-62).  The hash is FNV-1a over 64-bit
// tokens, computed by constexpr code only, so any compiler gives the same
// value for the same type.  Rules that differ only in the C++ spelling of an
// integer constant's type hash alike, as they evaluate alike.
#pragma once

#include <cstdint>
#include <type_traits>

#include "cellato/core/ast.hpp"

namespace cellato_b200::fingerprint {

namespace ast = cellato::ast;

constexpr uint64_t kOffset = 14695981039346656037ull;
constexpr uint64_t kPrime = 1099511628211ull;

constexpr uint64_t mix(uint64_t h, uint64_t token) {
    for (int i = 0; i < 8; ++i) {
        h ^= (token >> (8 * i)) & 0xffu;
        h *= kPrime;
    }
    return h;
}

template <auto V>
constexpr uint64_t value_token() {
    if constexpr (std::is_enum_v<decltype(V)>)
        return (uint64_t)(int64_t)static_cast<std::underlying_type_t<decltype(V)>>(V);
    else if constexpr (std::is_signed_v<decltype(V)>)
        return (uint64_t)(int64_t)V;
    else
        return (uint64_t)V;
}

// node<T>::hash(h) folds AST node T into h.  An AST node without a
// specialisation here fails to compile, as it would fail to lower.
template <typename T>
struct node;

enum tag : uint64_t {
    t_probability = 1, t_constant, t_state_constant, t_neighbor_at, t_moore, t_von_neumann, t_margolus,
    t_margolus_180, t_count, t_has_bit, t_if_then_else, t_and, t_or, t_not, t_bit_and, t_bit_or, t_plus,
    t_alternate, t_modulo, t_equals, t_greater, t_less, t_not_equals
};

template <uint64_t N, uint64_t D, uint64_t S>
struct node<ast::probability<N, D, S>> {
    static constexpr uint64_t hash(uint64_t h) { return mix(mix(mix(mix(h, t_probability), N), D), S); }
};
template <auto V>
struct node<ast::constant<V>> {
    static constexpr uint64_t hash(uint64_t h) { return mix(mix(h, t_constant), value_token<V>()); }
};
template <auto V>
struct node<ast::state_constant<V>> {
    static constexpr uint64_t hash(uint64_t h) { return mix(mix(h, t_state_constant), value_token<V>()); }
};
template <int X, int Y>
struct node<ast::neighbor_at<X, Y>> {
    static constexpr uint64_t hash(uint64_t h) {
        return mix(mix(mix(h, t_neighbor_at), (uint64_t)(int64_t)X), (uint64_t)(int64_t)Y);
    }
};
template <>
struct node<ast::moore_8_neighbors> {
    static constexpr uint64_t hash(uint64_t h) { return mix(h, t_moore); }
};
template <>
struct node<ast::von_neumann_4_neighbors> {
    static constexpr uint64_t hash(uint64_t h) { return mix(h, t_von_neumann); }
};
template <>
struct node<ast::margolus_alternating_neighborhood> {
    static constexpr uint64_t hash(uint64_t h) { return mix(h, t_margolus); }
};
template <>
struct node<ast::margolus_180_neighbor> {
    static constexpr uint64_t hash(uint64_t h) { return mix(h, t_margolus_180); }
};
template <typename C, typename N>
struct node<ast::count_neighbors<C, N>> {
    static constexpr uint64_t hash(uint64_t h) { return node<N>::hash(node<C>::hash(mix(h, t_count))); }
};
template <typename V, int B>
struct node<ast::has_bit_set<V, B>> {
    static constexpr uint64_t hash(uint64_t h) { return mix(node<V>::hash(mix(h, t_has_bit)), (uint64_t)B); }
};
template <typename C, typename T, typename E>
struct node<ast::if_then_else<C, T, E>> {
    static constexpr uint64_t hash(uint64_t h) {
        return node<E>::hash(node<T>::hash(node<C>::hash(mix(h, t_if_then_else))));
    }
};
template <typename V>
struct node<ast::not_<V>> {
    static constexpr uint64_t hash(uint64_t h) { return node<V>::hash(mix(h, t_not)); }
};
template <typename... A>
struct node<ast::alternate_algorithms<A...>> {
    static constexpr uint64_t hash(uint64_t h) {
        h = mix(mix(h, t_alternate), sizeof...(A));
        ((h = node<A>::hash(h)), ...);
        return h;
    }
};

// The two-operand nodes.
template <uint64_t Tag, typename L, typename R>
struct binary {
    static constexpr uint64_t hash(uint64_t h) { return node<R>::hash(node<L>::hash(mix(h, Tag))); }
};
template <typename L, typename R>
struct node<ast::and_<L, R>> : binary<t_and, L, R> {};
template <typename L, typename R>
struct node<ast::or_<L, R>> : binary<t_or, L, R> {};
template <typename L, typename R>
struct node<ast::bit_and_<L, R>> : binary<t_bit_and, L, R> {};
template <typename L, typename R>
struct node<ast::bit_or_<L, R>> : binary<t_bit_or, L, R> {};
template <typename L, typename R>
struct node<ast::plus<L, R>> : binary<t_plus, L, R> {};
template <typename L, typename R>
struct node<ast::modulo<L, R>> : binary<t_modulo, L, R> {};
template <typename L, typename R>
struct node<ast::equals<L, R>> : binary<t_equals, L, R> {};
template <typename L, typename R>
struct node<ast::greater_than<L, R>> : binary<t_greater, L, R> {};
template <typename L, typename R>
struct node<ast::less_than<L, R>> : binary<t_less, L, R> {};
template <typename L, typename R>
struct node<ast::not_equals<L, R>> : binary<t_not_equals, L, R> {};

template <typename Dict, int... I>
constexpr uint64_t dictionary_hash(uint64_t h, std::integer_sequence<int, I...>) {
    h = mix(mix(h, (uint64_t)Dict::number_of_values), (uint64_t)Dict::needed_bits);
    ((h = mix(h, (uint64_t)(int64_t)Dict::index_to_state(I))), ...);
    return h;
}

// The fingerprint of a Cellato config (its `algorithm` and `state_dictionary`).
template <typename Config>
constexpr uint64_t of() {
    using dict = typename Config::state_dictionary;
    const uint64_t h = node<typename Config::algorithm>::hash(kOffset);
    return dictionary_hash<dict>(h, std::make_integer_sequence<int, (int)dict::number_of_values>{});
}

} // namespace cellato_b200::fingerprint
