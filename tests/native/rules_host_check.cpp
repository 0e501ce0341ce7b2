// Host-side check of the word-wide rule networks in cb2_rules.cuh.
// Steps a toroidal bit-plane grid one generation with the same
// indicator / hagg / next structure the GPU strip kernel uses, for random
// grids, and prints the resulting planes so the Python test can compare them
// with the oracle.  Usage: rules_host_check <automaton> <x> <y> <steps> < planes > planes
#include <cstdint>
#include <cstdio>
#include <cstdlib>
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

int main(int argc, char** argv) {
    if (argc != 5) return 1;
    int aut = atoi(argv[1]), x = atoi(argv[2]), y = atoi(argv[3]), steps = atoi(argv[4]);
    switch (aut) {
    case 0: return run<cb2::game_of_life>(x, y, steps);
    case 1: return run<cb2::wire>(x, y, steps);
    case 2: return run<cb2::excitable>(x, y, steps);
    }
    return 1;
}
