// cb2_ast.cuh -- lowers a Cellato DSL rule (the type-level AST of
// core/ast.hpp) to word-wide bit-sliced device code for the strip kernels.
//
// The hand-written networks of cb2_rules.cuh cover the three headline
// automata.  Every other rule -- a bundled automaton or a user's -- runs
// through ast_rule<Config>: its window per row is the west / centre / east
// word of every bit-plane (3P words), and its next() evaluates the AST over
// the 3x3 window of those words, 32 cells at a time.  A node's value is a
// bit-sliced unsigned integer, bv<N>: N words, word i holding bit i of the
// value of each of the 32 cells.  The semantics are those of the reference's
// per-cell evaluator (evaluators/standard.hpp), which its bit-plane evaluator
// (evaluators/bit_planes.hpp) reproduces word-wide:
//
//   constant<V>                V (unsigned)
//   state_constant<S>          the dictionary index of S (states are stored as indexes)
//   neighbor_at<dx, dy>        the state index of cell (x+dx, y+dy), |dx|, |dy| <= 1, torus
//   equals / not_equals        comparison of the zero-extended values
//   greater_than / less_than   unsigned comparison
//   and_ / or_ / not_          logical (a value is true when non-zero)
//   bit_and_ / bit_or_         bitwise
//   plus                       exact sum (one bit wider than the wider operand)
//   modulo<L, constant<2^k>>   low k bits (only powers of two, as the reference)
//   has_bit_set<V, b>          bit b of V
//   if_then_else<C, T, E>      T where C is true, else E
//   count_neighbors<T, moore_8_neighbors | von_neumann_4_neighbors>
//                              how many neighbours equal T (T evaluated at the centre)
//   count_neighbors<T, margolus_alternating_neighborhood>, margolus_180_neighbor
//                              the 2x2 block of the cell, whose origin moves by
//                              (1, 1) with the parity of the generation
//                              (evaluators/standard.hpp:196-286)
//   alternate_algorithms<E, O> E on even generations, O on odd ones
//   probability<N, D, S>       a Bernoulli(N/D) draw per cell from the
//                              reference's counter-based SplitMix64 stream keyed
//                              by (seed, S, generation, x / 64, y), sampled
//                              exactly (core/probability.hpp:12-160)
//
// Evaluation is lazy where it pays: a branch of if_then_else, and the right
// operand of and_ / or_, is evaluated with the mask of the cells where its
// value is used (cell_ctx::care), and a probability draw resolves only those
// cells.  A cell's draw depends on that cell's random bits alone, so every
// used value is the reference's; values outside the mask are never read.
//
// The result of the rule is a state index; its low P bits are the new planes.
#pragma once

#include <cstdint>
#include <type_traits>

#include "cellato/core/ast.hpp"

#include "cb2_rules.cuh"
#include "cb2_strip.cuh"

namespace cb2 {
namespace ast {

namespace A = cellato::ast;

template <int N>
struct bv {
    static_assert(N >= 1, "a value has at least one bit");
    uint32_t w[N];
};

constexpr int bit_width_of(unsigned long long v) { return v ? 1 + bit_width_of(v >> 1) : 0; }
constexpr int max_of(int a, int b) { return a > b ? a : b; }

template <int M, int N>
__device__ __forceinline__ bv<M> resize(const bv<N>& x) {
    bv<M> r;
#pragma unroll
    for (int i = 0; i < M; ++i) r.w[i] = i < N ? x.w[i] : 0u;
    return r;
}

template <int N>
__device__ __forceinline__ uint32_t truth(const bv<N>& x) {
    uint32_t r = x.w[0];
#pragma unroll
    for (int i = 1; i < N; ++i) r |= x.w[i];
    return r;
}

__device__ __forceinline__ bv<1> mask(uint32_t m) { return bv<1>{{m}}; }

template <unsigned long long V>
__device__ __forceinline__ auto const_value() {
    constexpr int N = max_of(1, bit_width_of(V));
    bv<N> r;
#pragma unroll
    for (int i = 0; i < N; ++i) r.w[i] = ((V >> i) & 1ull) ? 0xffffffffu : 0u;
    return r;
}

template <int Na, int Nb>
__device__ __forceinline__ uint32_t eq_mask(const bv<Na>& a, const bv<Nb>& b) {
    constexpr int N = max_of(Na, Nb);
    uint32_t e = 0xffffffffu;
#pragma unroll
    for (int i = 0; i < N; ++i) e &= ~((i < Na ? a.w[i] : 0u) ^ (i < Nb ? b.w[i] : 0u));
    return e;
}

// a > b, unsigned, from the most significant bit down.
template <int Na, int Nb>
__device__ __forceinline__ uint32_t gt_mask(const bv<Na>& a, const bv<Nb>& b) {
    constexpr int N = max_of(Na, Nb);
    uint32_t gt = 0, eq = 0xffffffffu;
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        const uint32_t x = i < Na ? a.w[i] : 0u, y = i < Nb ? b.w[i] : 0u;
        gt |= eq & x & ~y;
        eq &= ~(x ^ y);
    }
    return gt;
}

template <int Na, int Nb>
__device__ __forceinline__ bv<max_of(Na, Nb) + 1> add(const bv<Na>& a, const bv<Nb>& b) {
    constexpr int N = max_of(Na, Nb);
    bv<N + 1> r;
    uint32_t carry = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const uint32_t x = i < Na ? a.w[i] : 0u, y = i < Nb ? b.w[i] : 0u;
        r.w[i] = xor3(x, y, carry);
        carry = maj3(x, y, carry);
    }
    r.w[N] = carry;
    return r;
}

// The 3x3 window of a row triple: (west, centre, east) word of each plane
// for the rows above (a), at (m) and below (b) the cells.
template <int P>
struct window {
    const uint32_t (&a)[3 * P];
    const uint32_t (&m)[3 * P];
    const uint32_t (&b)[3 * P];

    template <int DX, int DY>
    __device__ __forceinline__ bv<P> at() const {
        static_assert(DX >= -1 && DX <= 1 && DY >= -1 && DY <= 1, "neighbour offsets are limited to radius 1");
        const uint32_t(&row)[3 * P] = DY < 0 ? a : (DY > 0 ? b : m);
        bv<P> r;
#pragma unroll
        for (int p = 0; p < P; ++p) r.w[p] = row[3 * p + DX + 1];
        return r;
    }
};

// ---- SplitMix64 Bernoulli draws (core/probability.hpp) ----------------------------------------
__device__ __forceinline__ uint64_t sm_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ull;

// The reference keys one 64-bit stream per (seed, stream, generation, group
// of 64 cells, row): mix(mix(mix(mix(mix(seed + golden) ^ stream) ^ t) ^ x/64) ^ y).
// All but the last mix are the same for every row of a level, so the strip
// kernels compute this "lane key" once per task and level (ast_rule::init_keys).
__device__ __forceinline__ uint64_t lane_key(uint64_t seed, uint64_t stream, int64_t t, int64_t xw) {
    uint64_t k = sm_mix(seed + kGolden);
    k = sm_mix(k ^ stream);
    k = sm_mix(k ^ (uint64_t)t);
    return sm_mix(k ^ (uint64_t)(xw >> 1));
}

// Random 32-bit words for the lane's cells: draw n of the row's stream is
// mix(key + (n + 1) * golden), and a 32-bit word takes its half of it.
struct word_stream {
    uint64_t key;
    uint64_t counter = 0;
    unsigned shift;
    __device__ __forceinline__ word_stream(uint64_t lane, const cell_ctx& c)
        : key(sm_mix(lane ^ (uint64_t)c.y)), shift((unsigned)(c.xw & 1) * 32u) {}
    __device__ __forceinline__ uint32_t next() {
        counter += kGolden;
        return (uint32_t)(sm_mix(key + counter) >> shift);
    }
};

// The same stream when this lane and lane^1 hold the two halves of one group
// of 64 cells (cell_ctx::paired): the lane of the low half computes the even
// draws, its partner the odd ones, and each sends the other the half it
// uses -- one mix per two draws instead of one per draw.  (Letting a lone
// lane draw both halves inside one shared path instead cost lightning-forest
// a sixth of its speed: the second draw issues on every lane.)
struct pair_stream {
    uint64_t key;
    uint64_t counter = 0;
    unsigned shift;
    __device__ __forceinline__ pair_stream(uint64_t lane, const cell_ctx& c)
        : key(sm_mix(lane ^ (uint64_t)c.y)), shift((unsigned)(c.xw & 1) * 32u) {}
    // Draws 2m and 2m+1 (this lane's halves); every lane of the warp calls it together.
    __device__ __forceinline__ void next2(uint32_t& d0, uint32_t& d1) {
        const bool high = shift != 0;
        const uint64_t z = sm_mix(key + counter + (high ? 2 : 1) * kGolden);
        const uint32_t mine = (uint32_t)(z >> shift);
        const uint32_t other = __shfl_xor_sync(kFullMask, (uint32_t)(z >> (32u - shift)), 1);
        counter += 2 * kGolden;
        d0 = high ? other : mine;
        d1 = high ? mine : other;
    }
};

constexpr uint64_t gcd_of(uint64_t a, uint64_t b) { return b ? gcd_of(b, a % b) : a; }

// Draws the dyadic sampler below takes for N/D.
template <uint64_t N, uint64_t D>
constexpr int dyadic_draws() {
    if constexpr (N == 0 || N == D)
        return 0;
    else if constexpr (N >= D - N)
        return 1 + dyadic_draws<N - (D - N), D>();
    else
        return 1 + dyadic_draws<N + N, D>();
}

// Lane b is 1 with probability N/D (D a power of two): compares the binary
// expansion of N/D with one fresh random digit per draw (draws[j] is digit j).
template <uint64_t N, uint64_t D, int J = 0, int M>
__device__ __forceinline__ uint32_t dyadic_draw(const uint32_t (&draws)[M]) {
    if constexpr (N == 0) {
        return 0u;
    } else if constexpr (N == D) {
        return 0xffffffffu;
    } else {
        const uint32_t zero_bits = ~draws[J];
        if constexpr (N >= D - N)
            return zero_bits | dyadic_draw<N - (D - N), D, J + 1>(draws);
        else
            return zero_bits & dyadic_draw<N + N, D, J + 1>(draws);
    }
}

// The threshold n/d in binary: after j digits the remainder is rem_after(j),
// and digit j is 1 when 2 * rem >= d (compared before doubling, so that no
// sum exceeds 2^64, as the reference does).
constexpr uint64_t rem_after(uint64_t n, uint64_t d, int j) {
    for (int i = 0; i < j; ++i) n = n >= d - n ? n - (d - n) : n + n;
    return n;
}

// Digits J.. of the threshold against bits[J..]: a cell still active where its
// random bit equals the digit; it turns 1 where the digit is 1 and its bit 0.
// Inactive cells are left alone, so no per-lane test is needed.
template <uint64_t n, uint64_t d, int J, int M>
__device__ __forceinline__ void ratio_digits(const uint32_t (&bits)[M], uint32_t& active, uint32_t& result) {
    if constexpr (J < M) {
        constexpr uint64_t r = rem_after(n, d, J);
        if constexpr (r >= d - r) {
            result |= active & ~bits[J];
            active &= bits[J];
        } else {
            active &= ~bits[J];
        }
        ratio_digits<n, d, J + 1>(bits, active, result);
    }
}

// ratio_digits for digits J .. E-1 only.
template <uint64_t n, uint64_t d, int J, int E, int M>
__device__ __forceinline__ void ratio_digits_to(const uint32_t (&bits)[M], uint32_t& active, uint32_t& result) {
    if constexpr (J < E) {
        constexpr uint64_t r = rem_after(n, d, J);
        if constexpr (r >= d - r) {
            result |= active & ~bits[J];
            active &= bits[J];
        } else {
            active &= ~bits[J];
        }
        ratio_digits_to<n, d, J + 1, E>(bits, active, result);
    }
}

template <uint64_t Num, uint64_t Den>
__device__ __forceinline__ uint32_t bernoulli_word(const cell_ctx& c, uint64_t lane) {
    static_assert(Den > 0 && Num <= Den, "a probability lies in [0, 1]");
    if constexpr (Num == 0) {
        return 0u;
    } else if constexpr (Num == Den) {
        return 0xffffffffu;
    } else {
        constexpr uint64_t g = gcd_of(Num, Den);
        constexpr uint64_t n = Num / g, d = Den / g;
        if constexpr ((d & (d - 1)) == 0) {
            constexpr int M = dyadic_draws<n, d>();
            uint32_t draws[M + (M & 1)];
            if (!__any_sync(kFullMask, c.care)) return 0u;  // no cell of the warp uses the draw
            if (c.paired) {  // warp-uniform
                pair_stream s(lane, c);
#pragma unroll
                for (int j = 0; j < M; j += 2) s.next2(draws[j], draws[j + 1]);
            } else {
                word_stream s(lane, c);
#pragma unroll
                for (int j = 0; j < M; ++j) draws[j] = s.next();
            }
            return dyadic_draw<n, d>(draws);
        } else {
            // Recurring expansion: draw until every lane has left the threshold.
            // The stream is counter-based, so the first draws are computed up front
            // as independent instructions and compared with digits known at compile
            // time; draws past the one that resolves the last lane are not used.
            // A warp of 1024 cells needs about 11 digits, so a pair, whose shuffles
            // make the tail dearer, computes 12 up front (8: lightning-forest 0.99
            // against 1.15 Tcell/s).  Only the cells that use the draw
            // (cell_ctx::care) need to leave the threshold; when none of the warp's
            // is left after 10 digits, the last two are not drawn (lightning-forest
            // at 16384^2: 0.96 -> 1.05 Tcell/s; a first check after 6 or 8 digits
            // gained less, 1.00 and 1.03).
            uint32_t active = c.care, result = 0;
            auto digit = [&](uint64_t& rem, uint32_t bits) {
                if (rem >= d - rem) {
                    rem -= d - rem;
                    result |= active & ~bits;
                    active &= bits;
                } else {
                    rem += rem;
                    active &= ~bits;
                }
            };
            if (c.paired) {  // warp-uniform: the pair's shuffles run on every lane
                constexpr int kFirst = 10, kAhead = 12;
                if (!__any_sync(kFullMask, active)) return 0u;
                uint32_t ahead[kAhead];
                pair_stream s(lane, c);
#pragma unroll
                for (int j = 0; j < kFirst; j += 2) s.next2(ahead[j], ahead[j + 1]);
                ratio_digits_to<n, d, 0, kFirst>(ahead, active, result);
                if (!__any_sync(kFullMask, active)) return result;
#pragma unroll
                for (int j = kFirst; j < kAhead; j += 2) s.next2(ahead[j], ahead[j + 1]);
                ratio_digits_to<n, d, kFirst, kAhead>(ahead, active, result);
                uint64_t rem = rem_after(n, d, kAhead);
                while (__any_sync(kFullMask, active)) {
                    uint32_t d0, d1;
                    s.next2(d0, d1);
                    if (active) digit(rem, d0);
                    if (active) digit(rem, d1);
                }
            } else {
                constexpr int kAhead = 8;
                uint32_t ahead[kAhead];
                word_stream s(lane, c);
#pragma unroll
                for (int j = 0; j < kAhead; ++j) ahead[j] = s.next();
                ratio_digits<n, d, 0>(ahead, active, result);
                uint64_t rem = rem_after(n, d, kAhead);
                while (active) digit(rem, s.next());
            }
            return result;
        }
    }
}

// ---- the probability streams of a rule -----------------------------------------------------------
// The distinct Stream values of the probability<N, D, Stream> nodes of an
// AST, in order of first appearance: ast_rule keeps one lane key per stream
// and level.
template <uint64_t... S>
struct stream_list {
    static constexpr int size = sizeof...(S);
};

template <class L, uint64_t S>
struct with_stream;
template <uint64_t... T, uint64_t S>
struct with_stream<stream_list<T...>, S> {
    using type = std::conditional_t<((T == S) || ...), stream_list<T...>, stream_list<T..., S>>;
};

template <class L, class M>
struct join_streams;
template <class L>
struct join_streams<L, stream_list<>> {
    using type = L;
};
template <class L, uint64_t S, uint64_t... Rest>
struct join_streams<L, stream_list<S, Rest...>> {
    using type = typename join_streams<typename with_stream<L, S>::type, stream_list<Rest...>>::type;
};

template <class... Ls>
struct join_all {
    using type = stream_list<>;
};
template <class L, class... Ls>
struct join_all<L, Ls...> {
    using type = typename join_streams<L, typename join_all<Ls...>::type>::type;
};

template <class Node>
struct streams_of {  // leaves: constants, neighbours, neighbourhood tags
    using type = stream_list<>;
};
template <uint64_t Num, uint64_t Den, uint64_t S>
struct streams_of<A::probability<Num, Den, S>> {
    using type = stream_list<S>;
};
template <class V, int B>
struct streams_of<A::has_bit_set<V, B>> {
    using type = typename streams_of<V>::type;
};
template <template <class...> class T, class... Args>
struct streams_of<T<Args...>> {
    using type = typename join_all<typename streams_of<Args>::type...>::type;
};

template <uint64_t S, uint64_t... T>
constexpr int slot_of(stream_list<T...>) {
    constexpr uint64_t v[] = {T..., 0};
    for (int i = 0; i < (int)sizeof...(T); ++i)
        if (v[i] == S) return i;
    return -1;
}

// Whether an AST branches on the parity of the generation
// (alternate_algorithms): the strip kernels then fix each level's parity at
// compile time, so the branch folds (traffic: 23 -> 33 Tcell/s).  The
// Margolus nodes also read the parity, but as masks and selects: fixing it
// there measured slower (critters 12.9 -> 11.9), so they do not count.
template <class Node>
struct reads_parity : std::false_type {};
template <class E, class O>
struct reads_parity<A::alternate_algorithms<E, O>> : std::true_type {};
template <class V, int B>
struct reads_parity<A::has_bit_set<V, B>> : reads_parity<V> {};
template <template <class...> class T, class... Args>
struct reads_parity<T<Args...>> : std::bool_constant<(reads_parity<Args>::value || ...)> {};

// A state dictionary that also names the rule's streams, so that the
// probability evaluator finds its stream's slot in cell_ctx::key.
template <class D, class Streams>
struct keyed_dict : D {
    using streams = Streams;
};

template <class D, class = void>
struct has_streams : std::false_type {};
template <class D>
struct has_streams<D, std::void_t<typename D::streams>> : std::true_type {};

// Lanes whose Margolus partner (in x) is the cell to their right, for
// generation parity `odd`: even cells at even generations, odd cells at odd.
__device__ __forceinline__ uint32_t margolus_right_lanes(int64_t t) { return (t & 1) ? 0xaaaaaaaau : 0x55555555u; }
// +1 if the Margolus partner row is below the cells, -1 if above.
__device__ __forceinline__ int margolus_dy(const cell_ctx& c) { return (((c.y ^ c.t) & 1) == 0) ? 1 : -1; }

// ---- node evaluation ------------------------------------------------------------------------------
template <class Dict, class E>
struct ev;

template <class Dict, auto V>
struct ev<Dict, A::constant<V>> {
    static_assert(V >= 0, "negative constants are not supported");
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>&, const cell_ctx&) {
        return const_value<(unsigned long long)V>();
    }
};

template <class Dict, auto S>
struct ev<Dict, A::state_constant<S>> {
    static constexpr int index = Dict::state_to_index(S);
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>&, const cell_ctx&) {
        return const_value<(unsigned long long)index>();
    }
};

template <class Dict, int DX, int DY>
struct ev<Dict, A::neighbor_at<DX, DY>> {
    template <int P>
    __device__ __forceinline__ static bv<P> eval(const window<P>& w, const cell_ctx&) {
        return w.template at<DX, DY>();
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::equals<L, R>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        return mask(eq_mask(ev<Dict, L>::eval(w, c), ev<Dict, R>::eval(w, c)));
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::not_equals<L, R>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        return mask(~eq_mask(ev<Dict, L>::eval(w, c), ev<Dict, R>::eval(w, c)));
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::greater_than<L, R>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        return mask(gt_mask(ev<Dict, L>::eval(w, c), ev<Dict, R>::eval(w, c)));
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::less_than<L, R>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        return mask(gt_mask(ev<Dict, R>::eval(w, c), ev<Dict, L>::eval(w, c)));
    }
};

// The right operand of and_ matters only where the left is true, of or_ only
// where it is false.
template <class Dict, class L, class R>
struct ev<Dict, A::and_<L, R>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        const uint32_t l = truth(ev<Dict, L>::eval(w, c));
        cell_ctx cr = c;
        cr.care = c.care & l;
        return mask(l & truth(ev<Dict, R>::eval(w, cr)));
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::or_<L, R>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        const uint32_t l = truth(ev<Dict, L>::eval(w, c));
        cell_ctx cr = c;
        cr.care = c.care & ~l;
        return mask(l | truth(ev<Dict, R>::eval(w, cr)));
    }
};

template <class Dict, class X>
struct ev<Dict, A::not_<X>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        return mask(~truth(ev<Dict, X>::eval(w, c)));
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::bit_and_<L, R>> {
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>& w, const cell_ctx& c) {
        const auto a = ev<Dict, L>::eval(w, c);
        const auto b = ev<Dict, R>::eval(w, c);
        constexpr int Na = sizeof(a.w) / 4, Nb = sizeof(b.w) / 4, N = max_of(Na, Nb);
        const bv<N> x = resize<N>(a), y = resize<N>(b);
        bv<N> r;
#pragma unroll
        for (int i = 0; i < N; ++i) r.w[i] = x.w[i] & y.w[i];
        return r;
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::bit_or_<L, R>> {
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>& w, const cell_ctx& c) {
        const auto a = ev<Dict, L>::eval(w, c);
        const auto b = ev<Dict, R>::eval(w, c);
        constexpr int Na = sizeof(a.w) / 4, Nb = sizeof(b.w) / 4, N = max_of(Na, Nb);
        const bv<N> x = resize<N>(a), y = resize<N>(b);
        bv<N> r;
#pragma unroll
        for (int i = 0; i < N; ++i) r.w[i] = x.w[i] | y.w[i];
        return r;
    }
};

template <class Dict, class L, class R>
struct ev<Dict, A::plus<L, R>> {
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>& w, const cell_ctx& c) {
        return add(ev<Dict, L>::eval(w, c), ev<Dict, R>::eval(w, c));
    }
};

template <class Dict, class L, auto M>
struct ev<Dict, A::modulo<L, A::constant<M>>> {
    static_assert(M > 0 && (M & (M - 1)) == 0, "only modulo by a power of two is supported");
    static constexpr int k = bit_width_of((unsigned long long)M) - 1;
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>& w, const cell_ctx& c) {
        const auto a = ev<Dict, L>::eval(w, c);
        if constexpr (k == 0) {
            return mask(0u);
        } else {
            return resize<k>(a);
        }
    }
};

template <class Dict, class X, int B>
struct ev<Dict, A::has_bit_set<X, B>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        const auto a = ev<Dict, X>::eval(w, c);
        constexpr int N = sizeof(a.w) / 4;
        if constexpr (B < N)
            return mask(a.w[B]);
        else
            return mask(0u);
    }
};

template <class Dict, class C, class T, class E>
struct ev<Dict, A::if_then_else<C, T, E>> {
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>& w, const cell_ctx& c) {
        const uint32_t m = truth(ev<Dict, C>::eval(w, c));
        cell_ctx ct = c, ce = c;  // each branch matters only where it is taken
        ct.care = c.care & m;
        ce.care = c.care & ~m;
        const auto a = ev<Dict, T>::eval(w, ct);
        const auto b = ev<Dict, E>::eval(w, ce);
        constexpr int N = max_of(sizeof(a.w) / 4, sizeof(b.w) / 4);
        const bv<N> x = resize<N>(a), y = resize<N>(b);
        bv<N> r;
#pragma unroll
        for (int i = 0; i < N; ++i) r.w[i] = (x.w[i] & m) | (y.w[i] & ~m);
        return r;
    }
};

template <class Dict, class Even, class Odd>
struct ev<Dict, A::alternate_algorithms<Even, Odd>> {
    template <int P>
    __device__ __forceinline__ static auto eval(const window<P>& w, const cell_ctx& c) {
        using Ta = decltype(ev<Dict, Even>::eval(w, c));
        using Tb = decltype(ev<Dict, Odd>::eval(w, c));
        constexpr int N = max_of(sizeof(Ta) / 4, sizeof(Tb) / 4);
        if (c.t & 1) return resize<N>(ev<Dict, Odd>::eval(w, c));  // the generation is warp-uniform
        return resize<N>(ev<Dict, Even>::eval(w, c));
    }
};

template <class Dict, uint64_t Num, uint64_t Den, uint64_t Stream>
struct ev<Dict, A::probability<Num, Den, Stream>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>&, const cell_ctx& c) {
        uint64_t lane;
        if constexpr (has_streams<Dict>::value) {
            constexpr int j = slot_of<Stream>(typename Dict::streams{});
            static_assert(j >= 0, "stream missing from the rule's stream list");
            lane = c.key ? c.key[j] : lane_key(c.seed, Stream, c.t, c.xw);
        } else {
            lane = lane_key(c.seed, Stream, c.t, c.xw);
        }
        return mask(bernoulli_word<Num, Den>(c, lane));
    }
};

// 3-input and 2-input sums of one-bit masks, as (sum, carry) words.
__device__ __forceinline__ void fa(uint32_t x, uint32_t y, uint32_t z, uint32_t& s, uint32_t& k) {
    s = xor3(x, y, z);
    k = maj3(x, y, z);
}

template <class Dict, class T>
struct ev<Dict, A::count_neighbors<T, A::moore_8_neighbors>> {
    template <int P>
    __device__ __forceinline__ static bv<4> eval(const window<P>& w, const cell_ctx& c) {
        const auto tgt = ev<Dict, T>::eval(w, c);
        const uint32_t nw = eq_mask(w.template at<-1, -1>(), tgt), n = eq_mask(w.template at<0, -1>(), tgt),
                       ne = eq_mask(w.template at<1, -1>(), tgt), we = eq_mask(w.template at<-1, 0>(), tgt),
                       ea = eq_mask(w.template at<1, 0>(), tgt), sw = eq_mask(w.template at<-1, 1>(), tgt),
                       s = eq_mask(w.template at<0, 1>(), tgt), se = eq_mask(w.template at<1, 1>(), tgt);
        uint32_t s_a, c_a, s_b, c_b;
        fa(nw, n, ne, s_a, c_a);
        fa(sw, s, se, s_b, c_b);
        const uint32_t s_m = we ^ ea, c_m = we & ea;
        uint32_t t0, k0, x, y;
        fa(s_a, s_m, s_b, t0, k0);  // weight 1
        fa(c_a, c_m, c_b, x, y);    // weight 2 (x) and 4 (y)
        bv<4> r;
        r.w[0] = t0;
        r.w[1] = x ^ k0;
        const uint32_t k1 = x & k0;
        r.w[2] = y ^ k1;
        r.w[3] = y & k1;
        return r;
    }
};

template <class Dict, class T>
struct ev<Dict, A::count_neighbors<T, A::von_neumann_4_neighbors>> {
    template <int P>
    __device__ __forceinline__ static bv<3> eval(const window<P>& w, const cell_ctx& c) {
        const auto tgt = ev<Dict, T>::eval(w, c);
        const uint32_t up = eq_mask(w.template at<0, -1>(), tgt), rt = eq_mask(w.template at<1, 0>(), tgt),
                       dn = eq_mask(w.template at<0, 1>(), tgt), lf = eq_mask(w.template at<-1, 0>(), tgt);
        uint32_t s1, c1;
        fa(up, rt, dn, s1, c1);
        bv<3> r;
        r.w[0] = s1 ^ lf;
        const uint32_t k = s1 & lf;
        r.w[1] = c1 ^ k;
        r.w[2] = c1 & k;
        return r;
    }
};

// "Any neighbour equals T" without building the count.
template <class Dict, class T, class Nb>
struct ev<Dict, A::greater_than<A::count_neighbors<T, Nb>, A::constant<0>>> {
    template <int P>
    __device__ __forceinline__ static bv<1> eval(const window<P>& w, const cell_ctx& c) {
        if constexpr (std::is_same_v<Nb, A::moore_8_neighbors>) {
            const auto tgt = ev<Dict, T>::eval(w, c);
            return mask(eq_mask(w.template at<-1, -1>(), tgt) | eq_mask(w.template at<0, -1>(), tgt) |
                        eq_mask(w.template at<1, -1>(), tgt) | eq_mask(w.template at<-1, 0>(), tgt) |
                        eq_mask(w.template at<1, 0>(), tgt) | eq_mask(w.template at<-1, 1>(), tgt) |
                        eq_mask(w.template at<0, 1>(), tgt) | eq_mask(w.template at<1, 1>(), tgt));
        } else {
            return mask(truth(ev<Dict, A::count_neighbors<T, Nb>>::eval(w, c)));
        }
    }
};

template <class Dict, class T>
struct ev<Dict, A::count_neighbors<T, A::margolus_alternating_neighborhood>> {
    template <int P>
    __device__ __forceinline__ static bv<3> eval(const window<P>& w, const cell_ctx& c) {
        const auto tgt = ev<Dict, T>::eval(w, c);
        const uint32_t right = margolus_right_lanes(c.t);
        const bool below = margolus_dy(c) > 0;  // uniform across the warp
        // the cell, its horizontal partner, and the same two in the partner row
        const uint32_t e_c = eq_mask(w.template at<0, 0>(), tgt);
        const uint32_t e_h = (eq_mask(w.template at<1, 0>(), tgt) & right) | (eq_mask(w.template at<-1, 0>(), tgt) & ~right);
        const uint32_t e_v = below ? eq_mask(w.template at<0, 1>(), tgt) : eq_mask(w.template at<0, -1>(), tgt);
        const uint32_t e_d = below ? (eq_mask(w.template at<1, 1>(), tgt) & right) | (eq_mask(w.template at<-1, 1>(), tgt) & ~right)
                                   : (eq_mask(w.template at<1, -1>(), tgt) & right) | (eq_mask(w.template at<-1, -1>(), tgt) & ~right);
        uint32_t s1, c1;
        fa(e_c, e_h, e_v, s1, c1);
        bv<3> r;
        r.w[0] = s1 ^ e_d;
        const uint32_t k = s1 & e_d;
        r.w[1] = c1 ^ k;
        r.w[2] = c1 & k;
        return r;
    }
};

template <class Dict>
struct ev<Dict, A::margolus_180_neighbor> {
    template <int P>
    __device__ __forceinline__ static bv<P> eval(const window<P>& w, const cell_ctx& c) {
        const uint32_t right = margolus_right_lanes(c.t);
        const bool below = margolus_dy(c) > 0;
        const bv<P> r_b = w.template at<1, 1>(), l_b = w.template at<-1, 1>();
        const bv<P> r_a = w.template at<1, -1>(), l_a = w.template at<-1, -1>();
        bv<P> r;
#pragma unroll
        for (int p = 0; p < P; ++p)
            r.w[p] = below ? (r_b.w[p] & right) | (l_b.w[p] & ~right) : (r_a.w[p] & right) | (l_a.w[p] & ~right);
        return r;
    }
};

} // namespace ast

// A DSL automaton (a Cellato config: algorithm + state_dictionary) as a
// window rule for the strip kernels.
template <class Config>
struct ast_rule {
    using dict = typename Config::state_dictionary;
    using streams = typename ast::streams_of<typename Config::algorithm>::type;
    static constexpr int P = dict::needed_bits;
    static constexpr int NH = 3 * P;  // (west, centre, east) word of each plane
    static constexpr bool kWindow = true;
    static constexpr bool kDraws = streams::size > 0;  // the rule draws random numbers
    static constexpr bool kParity = ast::reads_parity<typename Config::algorithm>::value;

    // The lane keys of one level (cell_ctx::key), one per stream.
    struct level_keys {
        uint64_t k[streams::size > 0 ? streams::size : 1];
    };
    __device__ __forceinline__ static void init_keys(level_keys& keys, int64_t t, int64_t xw, uint64_t seed) {
        init_keys(keys, t, xw, seed, streams{});
    }
    template <uint64_t... S>
    __device__ __forceinline__ static void init_keys(level_keys& keys, int64_t t, int64_t xw, uint64_t seed,
                                                     ast::stream_list<S...>) {
        int j = 0;
        ((keys.k[j++] = ast::lane_key(seed, S, t, xw)), ...);
    }

    __device__ __forceinline__ static void next_at(const uint32_t (&a)[NH], const uint32_t (&m)[NH],
                                                   const uint32_t (&b)[NH], uint32_t (&o)[P],
                                                   const cell_ctx& c) {
        const ast::window<P> w{a, m, b};
        const auto r = ast::ev<ast::keyed_dict<dict, streams>, typename Config::algorithm>::eval(w, c);
        constexpr int N = sizeof(r.w) / 4;
#pragma unroll
        for (int p = 0; p < P; ++p) o[p] = p < N ? r.w[p] : 0u;
    }
};

} // namespace cb2
