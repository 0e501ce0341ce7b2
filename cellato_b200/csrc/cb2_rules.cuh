// cb2_rules.cuh -- word-wide rule networks for the bundled automata.
//
// Every rule here is a bit-sliced boolean network over 32-bit words: bit i of
// a word is cell x0+i of one bit-plane (bit b of the cell's state-dictionary
// index).  The networks are written so that each line is one three-input
// logic operation (one LOP3 on the GPU).
//
// Structure shared by all rules (the "Moore census" shape):
//   indicator(state)      1 plane: cells equal to the counted state
//   hagg(l, c, r)         horizontal aggregate of a row's indicator and its
//                         left/right neighbours (sum as 2 planes, or OR)
//   next(a, m, b, centre) vertical combine of the aggregates of the rows
//                         above/at/below plus the centre state -> new state
// The census includes the centre cell.  That is exact for these rules:
//   * game of life: with T = live cells in the 3x3 block, next is alive iff
//     T == 3, or T == 4 and the centre is alive (B3/S23,
//     game_of_life/algorithm.hpp:36-50);
//   * wireworld: the head count only matters for a conductor centre, which is
//     not a head, so the 3x3 count equals the Moore count
//     (wire/algorithm.hpp:48-59);
//   * greenberg-hastings: "any excited neighbour" only matters for a
//     quiescent centre, which is not excited (excitable/algorithm.hpp:58-72).
// Dictionary indexes follow the reference configs: wire empty=0 head=1 tail=2
// conductor=3 (wire/config.hpp:21-24); excitable 0..7 (excitable/config.hpp:21-28).
#pragma once

#include <cstdint>
#include <type_traits>

#if defined(__CUDACC__)
#define CB2_HD __host__ __device__ __forceinline__
#else
#define CB2_HD inline
#endif

namespace cb2 {

// Cell x-1 for every bit of `c`, taking bit 31 of the word to the left.
CB2_HD uint32_t west_of(uint32_t left, uint32_t c) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_l(left, c, 1);
#else
    return (c << 1) | (left >> 31);
#endif
}

// Cell x+1 for every bit of `c`, taking bit 0 of the word to the right.
CB2_HD uint32_t east_of(uint32_t c, uint32_t right) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_r(c, right, 1);
#else
    return (c >> 1) | (right << 31);
#endif
}

// One three-input logic operation with truth table LUT: bit i of LUT is the
// result for a = bit 2 of i, b = bit 1, c = bit 0 (a = 0xF0, b = 0xCC,
// c = 0xAA give LUT back).  On the device it is emitted as one lop3.b32, so
// a network written with it keeps the operation count it is written with;
// the host evaluates the same table.
template <unsigned LUT>
CB2_HD uint32_t lop3(uint32_t a, uint32_t b, uint32_t c) {
#if defined(__CUDA_ARCH__)
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(LUT));
    return d;
#else
    uint32_t d = 0;
    for (unsigned i = 0; i < 8; ++i)
        if ((LUT >> i) & 1u) d |= ((i & 4u) ? a : ~a) & ((i & 2u) ? b : ~b) & ((i & 1u) ? c : ~c);
    return d;
#endif
}

CB2_HD uint32_t xor3(uint32_t a, uint32_t b, uint32_t c) { return a ^ b ^ c; }
CB2_HD uint32_t maj3(uint32_t a, uint32_t b, uint32_t c) { return (a & b) | (c & (a | b)); }

// 3x3 census as a bit-sliced sum of three 2-bit row sums (a, m, b), each
// 0..3.  Returns the low three bits of the total (0..9); bit 3 is never
// needed by the rules below (see each rule).
CB2_HD void census_sum(const uint32_t (&a)[2], const uint32_t (&m)[2], const uint32_t (&b)[2], uint32_t& t0,
                       uint32_t& t1, uint32_t& t2) {
    t0 = xor3(a[0], m[0], b[0]);
    uint32_t k0 = maj3(a[0], m[0], b[0]);  // carry into weight 2
    uint32_t x = xor3(a[1], m[1], b[1]);
    uint32_t y = maj3(a[1], m[1], b[1]);   // weight 4
    t1 = x ^ k0;
    t2 = y ^ (x & k0);
}

// Game of Life, P = 1 (dead=0, alive=1).
struct game_of_life {
    static constexpr int P = 1;   // bit-planes of state
    static constexpr int NH = 2;  // planes of the horizontal aggregate
    static constexpr int id = 0;
    static constexpr bool kWindow = false;  // census network (a window rule sees all planes)
    CB2_HD static uint32_t indicator(const uint32_t (&s)[P]) { return s[0]; }
    CB2_HD static void hagg(uint32_t l, uint32_t c, uint32_t r, uint32_t (&h)[NH]) {
        h[0] = lop3<0x96>(l, c, r);  // xor3
        h[1] = lop3<0xE8>(l, c, r);  // majority
    }
    // T == 3 -> alive; T == 4 -> keep centre; otherwise dead.  T <= 9, and the
    // dropped bit 3 cannot alias 3 (11) or 4 (12).
    CB2_HD static void next(const uint32_t (&a)[NH], const uint32_t (&m)[NH], const uint32_t (&b)[NH],
                            const uint32_t (&c)[P], uint32_t (&o)[P]) {
        uint32_t t0, t1, t2;
        census_sum(a, m, b, t0, t1, t2);
        uint32_t e = ~(t0 ^ t1) & (t0 ^ t2);  // (t0,t1,t2) is (1,1,0) or (0,0,1)
        o[0] = e & (t0 | c[0]);
    }
    // Rows in pairs: output rows r and r+1 share census rows r and r+1, so
    // their 2-bit counts are summed once (Q = 0..6, 4 LOP3) and each output
    // adds its third row's count z and tests the total in 5 LOP3:
    //   w  = (q1 ^ z1) ? ~q2 : q1 ^ q2     e  = ~(q1 ^ z1 ^ q0)
    //   g3 = LUT 0x41 (q0, z0, centre)     g4 = LUT 0x59 (q0, z0, e)
    //   alive = w & ~g3 & ~g4
    // (found by exhaustive search over LOP3 circuits, none of 4 gates exists;
    // checked against T == 3 | (T == 4 & centre) for every count and centre).
    // Per word and generation 4/2 + 5 + the row's 2 horizontal LOP3 = 9 LOP3
    // + 2 funnel shifts, against 10 + 2 row by row.
    static constexpr bool kPairs = true;
    // (written as explicit lop3: with C operators the compiler re-covers the
    // shared terms and issued 10.4 LOP3 per word-generation, as row by row)
    CB2_HD static void pair(const uint32_t (&x)[NH], const uint32_t (&y)[NH], uint32_t (&q)[3]) {
        const uint32_t k = lop3<0xC0>(x[0], y[0], x[0]);  // x0 & y0
        q[0] = lop3<0x3C>(x[0], y[0], x[0]);              // x0 ^ y0
        q[1] = lop3<0x96>(x[1], y[1], k);
        q[2] = lop3<0xE8>(x[1], y[1], k);
    }
    CB2_HD static void next_pair(const uint32_t (&q)[3], const uint32_t (&z)[NH], const uint32_t (&c)[P],
                                 uint32_t (&o)[P]) {
        const uint32_t w = lop3<0x56>(q[1], z[1], q[2]);
        const uint32_t e = lop3<0x69>(q[1], z[1], q[0]);
        const uint32_t g3 = lop3<0x41>(q[0], z[0], c[0]);
        const uint32_t g4 = lop3<0x59>(q[0], z[0], e);
        o[0] = lop3<0x10>(w, g3, g4);
    }
};

// Rules that also evaluate rows in pairs (R::kPairs: R::pair, R::next_pair).
template <class R, class = void>
struct has_pairs : std::false_type {};
template <class R>
struct has_pairs<R, std::void_t<decltype(R::kPairs)>> : std::bool_constant<R::kPairs> {};

#if defined(__CUDACC__)
// A 1 the compiler cannot see through (constant memory, set when the module
// loads); one per translation unit.
static __constant__ uint32_t cb2_unit = 1;
#endif
// x as a new value: a multiply by cb2_unit, on the FMA pipe that the networks
// leave idle.  A plane a rule passes on unchanged otherwise stays one value
// over several levels of the wavefront, and the registers of the unrolled
// levels cannot follow it (the shift-register Greenberg-Hastings network below
// needed a fourth register per level and word: 255 and spills at 16 levels
// per warp and two words per lane, 228 and none with fresh copies).  The batch
// kernels (one word per lane, eight levels per warp, ~120 registers) are not
// short of registers, so their translation units define CB2_PLAIN_COPIES and
// keep plain copies instead of the extra multiplies.
CB2_HD uint32_t fresh(uint32_t x) {
#if defined(__CUDA_ARCH__) && !defined(CB2_PLAIN_COPIES)
    return x * cb2_unit;
#else
    return x;
#endif
}

// WireWorld, P = 2 (empty=0, head=1, tail=2, conductor=3).  Ten LOP3 and
// two funnel shifts per word and generation, each written as one lop3.
struct wire {
    static constexpr int P = 2;
    static constexpr int NH = 2;
    static constexpr int id = 1;
    static constexpr bool kWindow = false;
    // head: s0 & ~s1
    CB2_HD static uint32_t indicator(const uint32_t (&s)[P]) { return lop3<0x30>(s[0], s[1], s[0]); }
    // the row's head count over (x-1, x, x+1) as two bits: xor3 and majority
    CB2_HD static void hagg(uint32_t l, uint32_t c, uint32_t r, uint32_t (&h)[NH]) {
        h[0] = lop3<0x96>(l, c, r);
        h[1] = lop3<0xE8>(l, c, r);
    }
    // head->tail, tail->conductor, conductor->head iff 1..2 head neighbours,
    // empty->empty.  With the three rows' counts a, m, b (0..3 each) the 3x3
    // count is S = p0 + 2*k0 + 2*x + 4*y for p0 = a0^m0^b0, k0 = maj(a0, m0,
    // b0), x = a1^m1^b1, y = maj(a1, m1, b1); the centre is included, which is
    // exact because only a conductor centre reads the count and it is not a
    // head.  S is 1 or 2 iff y == 0 and (p0 ? k0 == x == 0 : k0 != x).
    CB2_HD static void next(const uint32_t (&a)[NH], const uint32_t (&m)[NH], const uint32_t (&b)[NH],
                            const uint32_t (&c)[P], uint32_t (&o)[P]) {
        const uint32_t p0 = lop3<0x96>(a[0], m[0], b[0]);
        const uint32_t k0 = lop3<0xE8>(a[0], m[0], b[0]);
        const uint32_t x = lop3<0x96>(a[1], m[1], b[1]);
        const uint32_t y = lop3<0xE8>(a[1], m[1], b[1]);
        const uint32_t g = lop3<0x16>(p0, k0, x);      // p0 ? ~k0 & ~x : k0 ^ x
        const uint32_t one_or_two = lop3<0x30>(g, y, g);  // g & ~y
        o[0] = fresh(c[1]);
        // (c0 ^ c1) | (c0 & c1 & ~one_or_two): head -> tail (2), tail -> conductor (3), conductor -> 1 or 3
        o[1] = lop3<0x7C>(c[0], c[1], one_or_two);
    }
    // Rows in pairs (see game_of_life): the two shared rows' head counts x, y
    // become the planes of their sum Q that the test reads -- Q bit 0, [Q <= 1]
    // and Q bit 2 (Q bit 1 is not needed), 4 LOP3 -- and each output adds its
    // third row's count z: the count is 1 or 2 iff LUT 0x86 of (z1, [Q <= 1],
    // ~q0 & ~q2 & ~z0) (3-gate circuit found by exhaustive search, none of 2
    // exists; checked for every Q and z).  Per word and generation 1 + 2 +
    // 4/2 + 3 = 8 LOP3 + 2 funnel shifts, against 10 + 2 row by row.
    static constexpr bool kPairs = true;
    CB2_HD static void pair(const uint32_t (&x)[NH], const uint32_t (&y)[NH], uint32_t (&q)[3]) {
        const uint32_t k = lop3<0xC0>(x[0], y[0], x[0]);  // x0 & y0
        q[0] = lop3<0x3C>(x[0], y[0], x[0]);              // x0 ^ y0
        q[1] = lop3<0x01>(x[1], y[1], k);                 // Q <= 1
        q[2] = lop3<0xE8>(x[1], y[1], k);                 // Q bit 2
    }
    CB2_HD static void next_pair(const uint32_t (&q)[3], const uint32_t (&z)[NH], const uint32_t (&c)[P],
                                 uint32_t (&o)[P]) {
        const uint32_t g = lop3<0x01>(q[0], q[2], z[0]);
        const uint32_t one_or_two = lop3<0x86>(z[1], q[1], g);
        o[0] = fresh(c[1]);
        o[1] = lop3<0x7C>(c[0], c[1], one_or_two);
    }
};

// Greenberg-Hastings excitable medium, P = 3 (quiescent=0, excited=1,
// refractory 2..7).  Inside a launch a cell's three bits are a de Bruijn
// shift register instead of its dictionary index: the cycle q -> e -> r1 ->
// ... -> r6 -> q is the sequence of 3-bit windows of the cyclic word
// 00010111 (as s2 s1 s0: q=000 e=001 r1=010 r2=101 r3=011 r4=111 r5=110
// r6=100), so a generation moves s1 to s2 and s0 to s1 and computes one new
// s0.  Per word and generation that is 5 LOP3 + 2 funnel shifts against
// 7 + 2 on the dictionary indexes; the three planes are re-encoded as rows
// enter a launch and decoded as they are stored (3 LOP3 each way, once per
// launch of K generations).
struct excitable {
    static constexpr int P = 3;
    static constexpr int NH = 1;
    static constexpr int id = 2;
    static constexpr bool kWindow = false;
    static constexpr bool kCodec = true;
    // dictionary index bits (r2 r1 r0) -> shift register (s2 s1 s0)
    CB2_HD static void encode(uint32_t (&s)[P]) {
        const uint32_t r0 = s[0], r1 = s[1], r2 = s[2];
        s[0] = lop3<0x3A>(r2, r1, r0);
        s[1] = lop3<0x74>(r2, r1, r0);
        s[2] = lop3<0xE8>(r2, r1, r0);
    }
    // shift register (s2 s1 s0) -> dictionary index bits (r2 r1 r0)
    CB2_HD static void decode(uint32_t (&s)[P]) {
        const uint32_t s0 = s[0], s1 = s[1], s2 = s[2];
        s[0] = lop3<0xB2>(s2, s1, s0);
        s[1] = lop3<0x74>(s2, s1, s0);
        s[2] = lop3<0xD8>(s2, s1, s0);
    }
    // excited: s2 s1 s0 = 001
    CB2_HD static uint32_t indicator(const uint32_t (&s)[P]) { return lop3<0x10>(s[0], s[1], s[2]); }
    CB2_HD static void hagg(uint32_t l, uint32_t c, uint32_t r, uint32_t (&h)[NH]) { h[0] = lop3<0xFE>(l, c, r); }
    // 0 -> 1 iff any excited neighbour; s -> s+1 for 1..6; 7 -> 0.  The new s0
    // is "any" for q (000) and the sequence's next bit otherwise (1 after 010,
    // 011 and 101): s2 ? s0 & G : s0 ^ G with G = s0 ? ~s1 : s1 | any.
    CB2_HD static void next(const uint32_t (&a)[NH], const uint32_t (&m)[NH], const uint32_t (&b)[NH],
                            const uint32_t (&c)[P], uint32_t (&o)[P]) {
        const uint32_t any = lop3<0xFE>(a[0], m[0], b[0]);
        const uint32_t g = lop3<0x3E>(c[1], c[0], any);
        o[0] = lop3<0x86>(c[2], c[0], g);
        o[1] = fresh(c[0]);
        o[2] = fresh(c[1]);
    }
};

// Rules that keep their states in another encoding inside a launch
// (R::kCodec: R::encode as rows enter the first level, R::decode as finished
// rows are stored), so that grids in memory always hold dictionary indexes;
// the other rules work on the indexes themselves.
template <class R, class = void>
struct has_codec : std::false_type {};
template <class R>
struct has_codec<R, std::void_t<decltype(R::kCodec)>> : std::bool_constant<R::kCodec> {};

template <class R>
CB2_HD void encode_states(uint32_t (&s)[R::P]) {
    if constexpr (has_codec<R>::value) R::encode(s);
}
template <class R>
CB2_HD void decode_states(uint32_t (&s)[R::P]) {
    if constexpr (has_codec<R>::value) R::decode(s);
}

} // namespace cb2
