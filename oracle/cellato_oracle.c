/*
 * cellato_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement, on the CPU, of what Cellato computes on the bit-plane
 * hot path.  Only the test suite, the smoke check and the CPU-baseline leg of
 * the benchmark may load this library, and only as the checker.  The product
 * (libcellato_b200.so) never links, loads or calls it.
 *
 * Parity pin: every function here is checked against the reference itself,
 * compiled from its own headers into oracle/_ref/ (ref_shim.cpp), and against
 * the committed golden fixtures generated from that build (tests/golden/);
 * the probability sampler (orc_sample_ratio) against the reference's own
 * scripted-word known answers (tests/probability.hpp:69-110).
 *
 * Cell encoding: one uint8 per cell holding the state-dictionary index
 * (memory/state_dictionary.hpp:10-42).  For the three bundled automata used
 * here the dictionary index equals the enum value:
 *   0 game-of-life  P=1  dead=0 alive=1           (game_of_life/config.hpp:21)
 *   1 wire          P=2  empty=0 head=1 tail=2 conductor=3 (wire/config.hpp:21-24)
 *   2 excitable     P=3  quiescent=0 excited=1 refractory_1..6=2..7
 *                                                 (excitable/config.hpp:21-28)
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_GOL 0
#define ORC_WIRE 1
#define ORC_EXCITABLE 2

int orc_planes(int automaton) {
    switch (automaton) {
    case ORC_GOL: return 1;
    case ORC_WIRE: return 2;
    case ORC_EXCITABLE: return 3;
    default: return -1;
    }
}

/* ------------------------------------------------------------------------ */
/* Seeded input generator (SplitMix64 counter stream).                       */
/* Cell i (= y*X + x) draws z = mix(seed + (i+1)*gamma); u = z >> 11 is a    */
/* uniform 53-bit integer; the state is the first j with u < thr[j], else    */
/* nthr.  thr[] are cumulative probabilities scaled by 2^53 (exact ints).    */
/* ------------------------------------------------------------------------ */
static inline uint64_t orc_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t orc_splitmix64(uint64_t seed, uint64_t index) {
    return orc_mix64(seed + (index + 1) * 0x9E3779B97F4A7C15ull);
}

void orc_init_cells(uint8_t* cells, uint64_t n_cells, uint64_t seed, const uint64_t* thr, int nthr) {
    for (uint64_t i = 0; i < n_cells; ++i) {
        uint64_t u = orc_splitmix64(seed, i) >> 11;
        int s = 0;
        while (s < nthr && u >= thr[s]) ++s;
        cells[i] = (uint8_t)s;
    }
}

/* ------------------------------------------------------------------------ */
/* Scalar rules, one cell at a time (evaluators/standard.hpp semantics).     */
/* ------------------------------------------------------------------------ */

/* Moore count of `state` around (x, y) with toroidal wrap
 * (memory/interface.hpp:31-36; evaluators/standard.hpp:178-194). */
static inline int moore_count(const uint8_t* g, int64_t X, int64_t Y, int64_t x, int64_t y, uint8_t state) {
    int n = 0;
    for (int dy = -1; dy <= 1; ++dy) {
        int64_t yy = (y + dy + Y) % Y;
        for (int dx = -1; dx <= 1; ++dx) {
            if (dx == 0 && dy == 0) continue;
            int64_t xx = (x + dx + X) % X;
            n += g[yy * X + xx] == state;
        }
    }
    return n;
}

/* One generation on the standard layout.
 * game_of_life/algorithm.hpp:36-50, wire/algorithm.hpp:48-59,
 * excitable/algorithm.hpp:58-72. */
int orc_step_standard(int automaton, int64_t X, int64_t Y, const uint8_t* in, uint8_t* out) {
    for (int64_t y = 0; y < Y; ++y) {
        for (int64_t x = 0; x < X; ++x) {
            uint8_t c = in[y * X + x];
            uint8_t n;
            switch (automaton) {
            case ORC_GOL: {
                int k = moore_count(in, X, Y, x, y, 1);
                n = c == 1 ? (uint8_t)(k == 2 || k == 3) : (uint8_t)(k == 3);
                break;
            }
            case ORC_WIRE: {
                if (c == 1) n = 2;
                else if (c == 2) n = 3;
                else if (c == 3) {
                    int k = moore_count(in, X, Y, x, y, 1);
                    n = (k == 1 || k == 2) ? 1 : 3;
                } else n = 0;
                break;
            }
            case ORC_EXCITABLE: {
                if (c == 0) n = moore_count(in, X, Y, x, y, 1) > 0 ? 1 : 0;
                else if (c < 7) n = (uint8_t)(c + 1);
                else n = 0;
                break;
            }
            default: return -1;
            }
            out[y * X + x] = n;
        }
    }
    return 0;
}

/* Double-buffered loop of the CPU simple traverser (traversers/cpu/simple.hpp:59-84). */
int orc_run_standard(int automaton, int64_t X, int64_t Y, int64_t steps, uint8_t* cells) {
    if (orc_planes(automaton) < 0 || X <= 0 || Y <= 0 || steps < 0) return -1;
    uint8_t* tmp = (uint8_t*)malloc((size_t)(X * Y));
    if (!tmp) return -2;
    uint8_t* cur = cells;
    uint8_t* nxt = tmp;
    for (int64_t s = 0; s < steps; ++s) {
        orc_step_standard(automaton, X, Y, cur, nxt);
        uint8_t* t = cur; cur = nxt; nxt = t;
    }
    if (cur != cells) memcpy(cells, cur, (size_t)(X * Y));
    free(tmp);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Word-wide bit-plane stepper (evaluators/bit_planes.hpp semantics):        */
/* neighbour words formed by shift+merge (bit_planes.hpp:315-387), equality  */
/* masks per state (vector_int.hpp:473-493), ripple-carry neighbour count    */
/* (bit_planes.hpp:521-562), and lane-mask blends for if/then/else           */
/* (bit_planes.hpp:114-134).  Words are 32-bit; bit i of word xw is cell     */
/* xw*32+i, which is byte-identical to the reference's 64-bit word layout.   */
/* ------------------------------------------------------------------------ */
typedef uint32_t orc_word;

static inline orc_word eq_state(const orc_word* v, int P, int state) {
    orc_word m = ~(orc_word)0;
    for (int b = 0; b < P; ++b) m &= ((state >> b) & 1) ? v[b] : ~v[b];
    return m;
}

/* neighbor_at<dx,dy> of one plane word.  dx=+1 reads cell x+1 (bit i+1). */
static inline orc_word nb_word(const orc_word* plane, int64_t XW, int64_t Y, int64_t xw, int64_t y, int dx, int dy) {
    int64_t yy = (y + dy + Y) % Y;
    orc_word c = plane[yy * XW + xw];
    if (dx == 0) return c;
    orc_word s = plane[yy * XW + (xw + dx + XW) % XW];
    if (dx > 0) return (c >> 1) | (s << 31);
    return (c << 1) | (s >> 31);
}

int orc_step_bit_planes(int automaton, int64_t X, int64_t Y, const orc_word* in, orc_word* out) {
    int P = orc_planes(automaton);
    if (P < 0 || X % 32) return -1;
    int64_t XW = X / 32, plane = XW * Y;
    static const int dxs[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
    static const int dys[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
    int counted = 1; /* alive / electron_head / excited all have index 1 */
    for (int64_t y = 0; y < Y; ++y) {
        for (int64_t xw = 0; xw < XW; ++xw) {
            orc_word cur[3];
            for (int b = 0; b < P; ++b) cur[b] = in[b * plane + y * XW + xw];
            /* ripple-carry count of the 8 equality masks into 4 bit-planes */
            orc_word cnt[4] = {0, 0, 0, 0};
            orc_word any = 0;
            for (int k = 0; k < 8; ++k) {
                orc_word v[3];
                for (int b = 0; b < P; ++b) v[b] = nb_word(in + b * plane, XW, Y, xw, y, dxs[k], dys[k]);
                orc_word m = eq_state(v, P, counted);
                any |= m;
                orc_word carry = m;
                for (int b = 0; b < 4; ++b) {
                    orc_word t = cnt[b] & carry;
                    cnt[b] ^= carry;
                    carry = t;
                }
            }
            /* count == n as a lane mask */
#define CNT_EQ(n) (((n & 1) ? cnt[0] : ~cnt[0]) & ((n & 2) ? cnt[1] : ~cnt[1]) & \
                   ((n & 4) ? cnt[2] : ~cnt[2]) & ((n & 8) ? cnt[3] : ~cnt[3]))
            orc_word nxt[3] = {0, 0, 0};
            if (automaton == ORC_GOL) {
                orc_word alive = eq_state(cur, 1, 1);
                orc_word two_or_three = CNT_EQ(2) | CNT_EQ(3);
                nxt[0] = (alive & two_or_three) | (~alive & CNT_EQ(3));
            } else if (automaton == ORC_WIRE) {
                orc_word head = eq_state(cur, 2, 1), tail = eq_state(cur, 2, 2), cond = eq_state(cur, 2, 3);
                orc_word one_or_two = CNT_EQ(1) | CNT_EQ(2);
                /* blend chain, innermost first:
                 *   conductor -> (head=1 if 1-2 heads else conductor=3), else empty=0
                 *   tail -> conductor=3
                 *   head -> tail=2 */
                orc_word r0 = cond;                /* bit0 of 1 or 3 is set */
                orc_word r1 = cond & ~one_or_two;  /* bit1 set only for 3 */
                r0 = tail | (~tail & r0);
                r1 = tail | (~tail & r1);
                r0 = ~head & r0;
                r1 = head | (~head & r1);
                nxt[0] = r0;
                nxt[1] = r1;
            } else {
                orc_word q = eq_state(cur, 3, 0);
                orc_word r[3] = {0, 0, 0}; /* else branch: quiescent */
                for (int s = 6; s >= 1; --s) { /* elif chain, innermost first */
                    orc_word is = eq_state(cur, 3, s);
                    int to = s + 1;
                    for (int b = 0; b < 3; ++b) r[b] = (is & (((to >> b) & 1) ? ~0u : 0u)) | (~is & r[b]);
                }
                orc_word exc = any; /* count > 0 fast path, bit_planes.hpp:607-630 */
                r[0] = (q & exc) | (~q & r[0]);
                r[1] = ~q & r[1];
                r[2] = ~q & r[2];
                for (int b = 0; b < 3; ++b) nxt[b] = r[b];
            }
#undef CNT_EQ
            for (int b = 0; b < P; ++b) out[b * plane + y * XW + xw] = nxt[b];
        }
    }
    return 0;
}

int orc_run_bit_planes(int automaton, int64_t X, int64_t Y, int64_t steps, orc_word* planes) {
    int P = orc_planes(automaton);
    if (P < 0 || X % 32 || Y <= 0 || steps < 0) return -1;
    size_t words = (size_t)(P * (X / 32) * Y);
    orc_word* tmp = (orc_word*)malloc(words * sizeof(orc_word));
    if (!tmp) return -2;
    orc_word* cur = planes;
    orc_word* nxt = tmp;
    for (int64_t s = 0; s < steps; ++s) {
        orc_step_bit_planes(automaton, X, Y, cur, nxt);
        orc_word* t = cur; cur = nxt; nxt = t;
    }
    if (cur != planes) memcpy(planes, cur, words * sizeof(orc_word));
    free(tmp);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Checksum: 4x4 tiles of ceil(X/4) x ceil(Y/4) cells, uint64 sum of the     */
/* state VALUES per tile, row-major tile order (standard_grid.hpp:182-218).  */
/* values[i] maps dictionary index i to its enum value.                      */
/* ------------------------------------------------------------------------ */
void orc_checksum(const uint8_t* cells, int64_t X, int64_t Y, const int64_t* values, uint64_t out[16]) {
    int64_t tw = (X + 3) / 4, th = (Y + 3) / 4;
    for (int ty = 0; ty < 4; ++ty) {
        for (int tx = 0; tx < 4; ++tx) {
            int64_t x0 = tx * tw, y0 = ty * th;
            int64_t x1 = x0 + tw < X ? x0 + tw : X, y1 = y0 + th < Y ? y0 + th : Y;
            uint64_t sum = 0;
            for (int64_t y = y0; y < y1; ++y)
                for (int64_t x = x0; x < x1; ++x) sum += (uint64_t)values[cells[y * X + x]];
            out[ty * 4 + tx] = sum;
        }
    }
}

/* The same checksum computed from bit planes (32-bit words, P planes of Y   */
/* rows of X/32 words), for grids too large to hold one byte per cell: each  */
/* word adds popcount(minterm(state) & tile columns) * value for each state. */
/* X must be a multiple of 32.                                               */
void orc_checksum_planes(const orc_word* planes, int64_t X, int64_t Y, int P, const int64_t* values,
                         uint64_t out[16]) {
    int64_t tw = (X + 3) / 4, th = (Y + 3) / 4, XW = X / 32, plane = XW * Y;
    memset(out, 0, 16 * sizeof(uint64_t));
    for (int64_t y = 0; y < Y; ++y) {
        int ty = (int)(y / th);
        for (int64_t xw = 0; xw < XW; ++xw) {
            orc_word v[8];
            for (int b = 0; b < P; ++b) v[b] = planes[b * plane + y * XW + xw];
            for (int tx = 0; tx < 4; ++tx) {
                int64_t x0 = tx * tw, x1 = x0 + tw < X ? x0 + tw : X;
                int64_t lo = x0 > xw * 32 ? x0 - xw * 32 : 0, hi = x1 < xw * 32 + 32 ? x1 - xw * 32 : 32;
                if (lo >= hi) continue;
                orc_word cols = (hi - lo == 32) ? ~(orc_word)0 : ((((orc_word)1 << (hi - lo)) - 1) << lo);
                for (int s = 0; s < (1 << P); ++s) {
                    uint64_t n = (uint64_t)__builtin_popcount(eq_state(v, P, s) & cols);
                    out[ty * 4 + tx] += n * (uint64_t)values[s];
                }
            }
        }
    }
}

/* orc_init_cells written straight into bit planes (same cell stream: cell   */
/* y*X + x draws index y*X + x), for grids too large for a byte per cell;    */
/* rows [row_first, row_first + row_count) only, so threads can share it.   */
int orc_init_bit_planes_rows(orc_word* planes, int64_t X, int64_t Y, int P, uint64_t seed, const uint64_t* thr,
                             int nthr, int64_t row_first, int64_t row_count) {
    if (X % 32 || P < 1 || P > 8 || row_first < 0 || row_count < 0 || row_first + row_count > Y) return -1;
    int64_t XW = X / 32, plane = XW * Y;
    for (int64_t y = row_first; y < row_first + row_count; ++y)
        for (int64_t xw = 0; xw < XW; ++xw) {
            orc_word w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int i = 0; i < 32; ++i) {
                uint64_t u = orc_splitmix64(seed, (uint64_t)(y * X + xw * 32 + i)) >> 11;
                int s = 0;
                while (s < nthr && u >= thr[s]) ++s;
                for (int b = 0; b < P; ++b) w[b] |= (orc_word)((s >> b) & 1) << i;
            }
            for (int b = 0; b < P; ++b) planes[b * plane + y * XW + xw] = w[b];
        }
    return 0;
}

int orc_init_bit_planes(orc_word* planes, int64_t X, int64_t Y, int P, uint64_t seed, const uint64_t* thr,
                        int nthr) {
    return orc_init_bit_planes_rows(planes, X, Y, P, seed, thr, nthr, 0, Y);
}

/* ------------------------------------------------------------------------ */
/* Layout packing (host byte images of the reference's grids).               */
/* ------------------------------------------------------------------------ */

/* bit_planes (memory/bit_planes_grid.hpp:234-270): plane b is Y rows of X/8
 * bytes; cell x of row y is bit (x % 8) of byte x/8.  Identical bytes for
 * 32- and 64-bit words on a little-endian host. */
int orc_pack_bit_planes(const uint8_t* cells, int64_t X, int64_t Y, int P, uint8_t* out) {
    if (X % 8) return -1;
    int64_t rb = X / 8, plane = rb * Y;
    memset(out, 0, (size_t)(plane * P));
    for (int64_t y = 0; y < Y; ++y)
        for (int64_t x = 0; x < X; ++x) {
            uint8_t s = cells[y * X + x];
            for (int b = 0; b < P; ++b)
                if ((s >> b) & 1) out[b * plane + y * rb + x / 8] |= (uint8_t)(1u << (x % 8));
        }
    return 0;
}

int orc_unpack_bit_planes(const uint8_t* in, int64_t X, int64_t Y, int P, uint8_t* cells) {
    if (X % 8) return -1;
    int64_t rb = X / 8, plane = rb * Y;
    for (int64_t y = 0; y < Y; ++y)
        for (int64_t x = 0; x < X; ++x) {
            uint8_t s = 0;
            for (int b = 0; b < P; ++b) s |= (uint8_t)(((in[b * plane + y * rb + x / 8] >> (x % 8)) & 1) << b);
            cells[y * X + x] = s;
        }
    return 0;
}

/* bit_array (memory/bit_array_grid.hpp:300-321): cells_per_word = W / P
 * whole states per W-bit word, cell i (= y*X + x) at word i/cpw, bit
 * (i % cpw) * P.  Words are stored little-endian. */
int orc_pack_bit_array(const uint8_t* cells, int64_t X, int64_t Y, int P, int W, uint8_t* out) {
    int cpw = W / P;
    if (X % cpw) return -1;
    int64_t n = X * Y, words = n / cpw;
    memset(out, 0, (size_t)(words * (W / 8)));
    for (int64_t i = 0; i < n; ++i) {
        int64_t w = i / cpw;
        int off = (int)(i % cpw) * P;
        for (int b = 0; b < P; ++b)
            if ((cells[i] >> b) & 1) {
                int bit = off + b;
                out[w * (W / 8) + bit / 8] |= (uint8_t)(1u << (bit % 8));
            }
    }
    return 0;
}

int orc_unpack_bit_array(const uint8_t* in, int64_t X, int64_t Y, int P, int W, uint8_t* cells) {
    int cpw = W / P;
    if (X % cpw) return -1;
    int64_t n = X * Y;
    for (int64_t i = 0; i < n; ++i) {
        int64_t w = i / cpw;
        int off = (int)(i % cpw) * P;
        uint8_t s = 0;
        for (int b = 0; b < P; ++b) {
            int bit = off + b;
            s |= (uint8_t)(((in[w * (W / 8) + bit / 8] >> (bit % 8)) & 1) << b);
        }
        cells[i] = s;
    }
    return 0;
}

/* tiled_bit_planes (memory/tiled_bit_planes_grid.hpp:244-287): each W-bit
 * word is an 8 x (W/8) tile; cell (x, y) sits in word (x/8, y/(W/8)) at bit
 * (x%8) + 8*(y%(W/8)).  Plane-major, tile words row-major. */
int orc_pack_tiled(const uint8_t* cells, int64_t X, int64_t Y, int P, int W, uint8_t* out) {
    int th = W / 8;
    if (X % 8 || Y % th) return -1;
    int64_t XT = X / 8, YT = Y / th, plane = XT * YT * (W / 8);
    memset(out, 0, (size_t)(plane * P));
    for (int64_t y = 0; y < Y; ++y)
        for (int64_t x = 0; x < X; ++x) {
            int64_t word = (y / th) * XT + x / 8;
            int bit = (int)(x % 8) + 8 * (int)(y % th);
            for (int b = 0; b < P; ++b)
                if ((cells[y * X + x] >> b) & 1) out[b * plane + word * (W / 8) + bit / 8] |= (uint8_t)(1u << (bit % 8));
        }
    return 0;
}

int orc_unpack_tiled(const uint8_t* in, int64_t X, int64_t Y, int P, int W, uint8_t* cells) {
    int th = W / 8;
    if (X % 8 || Y % th) return -1;
    int64_t XT = X / 8, YT = Y / th, plane = XT * YT * (W / 8);
    for (int64_t y = 0; y < Y; ++y)
        for (int64_t x = 0; x < X; ++x) {
            int64_t word = (y / th) * XT + x / 8;
            int bit = (int)(x % 8) + 8 * (int)(y % th);
            uint8_t s = 0;
            for (int b = 0; b < P; ++b) s |= (uint8_t)(((in[b * plane + word * (W / 8) + bit / 8] >> (bit % 8)) & 1) << b);
            cells[y * X + x] = s;
        }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Exact Bernoulli(num/den) sampling of probability<N, D, S>                 */
/* (core/probability.hpp:27-87).  Lane b of the result is 1 with             */
/* probability num/den; digit j of the comparison is bit b of words[j].      */
/* A power-of-two denominator compares its finite binary expansion with one  */
/* fresh word per digit (sample_dyadic, :27-43); any other ratio draws until */
/* every active lane has left the threshold (sample_ratio, :45-87), so no    */
/* precision is fixed.  Lanes outside `active` are never set.  lane_bits is  */
/* the word width (8, 16, 32 or 64); *used returns the words consumed, or -1 */
/* when `words` ran out first.                                               */
/* ------------------------------------------------------------------------ */
static uint64_t orc_gcd(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t r = a % b;
        a = b;
        b = r;
    }
    return a;
}

static uint64_t orc_dyadic(uint64_t num, uint64_t den, const uint64_t* words, int nwords, uint64_t mask, int* used) {
    if (num == 0) return 0;
    if (num == den) return mask;
    if (*used < 0 || *used >= nwords) {
        *used = -1;
        return 0;
    }
    const uint64_t zero_bits = ~words[(*used)++] & mask;
    if (num >= den - num) return zero_bits | orc_dyadic(num - (den - num), den, words, nwords, mask, used);
    return zero_bits & orc_dyadic(num + num, den, words, nwords, mask, used);
}

uint64_t orc_sample_ratio(uint64_t num, uint64_t den, const uint64_t* words, int nwords, uint64_t active,
                          int lane_bits, int* used) {
    const uint64_t mask = lane_bits >= 64 ? ~0ull : ((1ull << lane_bits) - 1);
    *used = 0;
    active &= mask;
    if (den == 0 || num > den) {
        *used = -1;
        return 0;
    }
    if (num == 0) return 0;
    if (num == den) return active;
    const uint64_t g = orc_gcd(num, den);
    const uint64_t n = num / g, d = den / g;
    if (active == 0) return 0;
    if ((d & (d - 1)) == 0) return active & orc_dyadic(n, d, words, nwords, mask, used);
    uint64_t result = 0, rem = n;
    while (active) {
        if (*used >= nwords) {
            *used = -1;
            return result;
        }
        const uint64_t bits = words[(*used)++] & mask;
        if (rem >= d - rem) { /* digit 1, compared before doubling: no overflow */
            rem -= d - rem;
            result |= active & ~bits;
            active &= bits;
        } else {
            rem += rem;
            active &= ~bits;
        }
    }
    return result;
}
