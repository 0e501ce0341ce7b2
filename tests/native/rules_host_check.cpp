// Host-side check of the word-wide rule networks in cb2_rules.cuh.
// Steps a toroidal bit-plane grid one generation with the same
// indicator / hagg / next structure the GPU strip kernel uses, for random
// grids, and prints the resulting planes so the Python test can compare them
// with the oracle.  Usage: rules_host_check <automaton> <x> <y> <steps> < planes > planes
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../cellato_b200/csrc/cb2_rules.cuh"

template <class R>
static void step(const std::vector<uint32_t>& in, std::vector<uint32_t>& out, int xw, int y) {
    const size_t plane = (size_t)xw * y;
    auto ind = [&](int r, int c) {
        uint32_t s[R::P];
        r = (r + y) % y;
        c = (c + xw) % xw;
        for (int p = 0; p < R::P; ++p) s[p] = in[p * plane + (size_t)r * xw + c];
        return R::indicator(s);
    };
    auto agg = [&](int r, int c, uint32_t (&h)[R::NH]) {
        R::hagg(cb2::west_of(ind(r, c - 1), ind(r, c)), ind(r, c), cb2::east_of(ind(r, c), ind(r, c + 1)), h);
    };
    for (int r = 0; r < y; ++r)
        for (int c = 0; c < xw; ++c) {
            uint32_t a[R::NH], m[R::NH], b[R::NH], s[R::P], o[R::P];
            agg(r - 1, c, a);
            agg(r, c, m);
            agg(r + 1, c, b);
            for (int p = 0; p < R::P; ++p) s[p] = in[p * plane + (size_t)r * xw + c];
            if constexpr (cb2::has_pairs<R>::value) {
                // the kernels' pair path: even rows pair with the row below and add
                // the row above, odd rows pair with the row above and add the row below
                uint32_t q[3];
                if (r % 2 == 0) {
                    R::pair(m, b, q);
                    R::next_pair(q, a, s, o);
                } else {
                    R::pair(a, m, q);
                    R::next_pair(q, b, s, o);
                }
            } else {
                R::next(a, m, b, s, o);
            }
            for (int p = 0; p < R::P; ++p) out[p * plane + (size_t)r * xw + c] = o[p];
        }
}

template <class R>
static int run(int x, int y, int steps) {
    int xw = x / 32;
    std::vector<uint32_t> a((size_t)R::P * xw * y), b(a.size());
    if (fread(a.data(), 4, a.size(), stdin) != a.size()) return 2;
    // the kernels' working encoding of the states (cb2::encode_states), as a launch enters and leaves it
    auto recode = [&](bool enc) {
        const size_t plane = (size_t)xw * y;
        for (size_t w = 0; w < plane; ++w) {
            uint32_t s[R::P];
            for (int p = 0; p < R::P; ++p) s[p] = a[p * plane + w];
            if (enc)
                cb2::encode_states<R>(s);
            else
                cb2::decode_states<R>(s);
            for (int p = 0; p < R::P; ++p) a[p * plane + w] = s[p];
        }
    };
    recode(true);
    for (int s = 0; s < steps; ++s) {
        step<R>(a, b, xw, y);
        a.swap(b);
    }
    recode(false);
    fwrite(a.data(), 4, a.size(), stdout);
    return 0;
}

// Exhaustive check of a rule's pair evaluation (cb2::has_pairs): every
// combination of the three census rows' 3-cell patterns and the centre state,
// one combination per bit of the words, against next() on the same rows, for
// both ways the kernels pair rows (the shared rows with the one above or below).
template <class R>
static int check_pairs(const char* name) {
    if constexpr (cb2::has_pairs<R>::value) {
        // 3 rows x 3 cells of indicator bits and P centre planes: 9 + P bits per case
        constexpr int kBits = 9 + R::P;
        long bad = 0, cases = 0;
        for (long base = 0; base < (1L << kBits); base += 32) {
            uint32_t cell[9] = {}, cen[R::P] = {};
            for (int b = 0; b < 32 && base + b < (1L << kBits); ++b) {
                const long v = base + b;
                for (int k = 0; k < 9; ++k) cell[k] |= (uint32_t)((v >> k) & 1) << b;
                for (int p = 0; p < R::P; ++p) cen[p] |= (uint32_t)((v >> (9 + p)) & 1) << b;
            }
            // row r's aggregate of its three indicator cells (the kernels' hagg)
            uint32_t h[3][R::NH];
            for (int r = 0; r < 3; ++r) R::hagg(cell[3 * r], cell[3 * r + 1], cell[3 * r + 2], h[r]);
            uint32_t want[R::P], got_lo[R::P], got_hi[R::P], q[3];
            R::next(h[0], h[1], h[2], cen, want);
            R::pair(h[1], h[2], q);  // the output pairs its own row with the row below
            R::next_pair(q, h[0], cen, got_lo);
            R::pair(h[0], h[1], q);  // ... or with the row above
            R::next_pair(q, h[2], cen, got_hi);
            const uint32_t live = base + 32 <= (1L << kBits) ? 0xffffffffu : (1u << ((1L << kBits) - base)) - 1;
            for (int p = 0; p < R::P; ++p) {
                uint32_t diff = ((want[p] ^ got_lo[p]) | (want[p] ^ got_hi[p])) & live;
                bad += __builtin_popcount(diff);
            }
            cases += __builtin_popcount(live);
        }
        printf("%s pairs: %ld cases, %ld mismatches\n", name, cases, bad);
        return bad ? 3 : 0;
    } else {
        printf("%s evaluates no pairs\n", name);
        return 0;
    }
}

int main(int argc, char** argv) {
    if (argc == 2 && std::string(argv[1]) == "pairs")
        return check_pairs<cb2::game_of_life>("game-of-life") | check_pairs<cb2::wire>("wire") |
               check_pairs<cb2::excitable>("excitable");
    if (argc != 5) return 1;
    int aut = atoi(argv[1]), x = atoi(argv[2]), y = atoi(argv[3]), steps = atoi(argv[4]);
    switch (aut) {
    case 0: return run<cb2::game_of_life>(x, y, steps);
    case 1: return run<cb2::wire>(x, y, steps);
    case 2: return run<cb2::excitable>(x, y, steps);
    }
    return 1;
}
