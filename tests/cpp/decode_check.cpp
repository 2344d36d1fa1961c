// Host build of the library's site decode (lattice.cuh): the multiply-shift
// division by the chain extents against plain division.
//   * div_by for every divisor 2..4096 on dividends spread over [0, 2^31) and
//     on every value near multiples of the divisor;
//   * decode of every site of a set of lattice shapes (odd, even, powers of two,
//     the 48^3 x 96 workload's extents) against % and /;
//   * on the same shapes, every site's neighbour index along each direction at
//     steps -2..2 from nb (dynamically indexed) and nb_sel (selects) against the
//     index of the wrapped coordinates.
// Prints "ok" and exits 0, or prints the first mismatch and exits 1.
#include <cstdio>
#include <cstdint>

#include "../../mag_b200/csrc/lattice.cuh"

using namespace magb;

static int check_divisor(unsigned d) {
    unsigned m;
    int sh;
    set_divisor(d, m, sh);
    auto one = [&](unsigned n) {
        if (div_by(n, m, sh) != n / d) {
            std::printf("div_by(%u, d=%u) = %u, expected %u\n", n, d, div_by(n, m, sh), n / d);
            return 1;
        }
        return 0;
    };
    for (unsigned n = 0; n < 70000; n++)
        if (one(n)) return 1;
    for (uint64_t n = 0; n < (1ull << 31); n += 982451u)
        if (one((unsigned)n)) return 1;
    for (uint64_t k = 1; k * d < (1ull << 31); k = k * 3 + 1)
        for (int e = -2; e <= 2; e++)
            if (one((unsigned)(k * d + e))) return 1;
    return one((1u << 31) - 1);
}

static int check_lattice(int L0, int L1, int L2, int L3) {
    ChainInfo ci{};
    const int L[4] = {L0, L1, L2, L3};
    long V = 1;
    for (int d = 0; d < 4; d++) {
        ci.L[d] = L[d];
        ci.stride[d] = (int)V;
        V *= L[d];
    }
    set_divisors(ci);
    ci.V = (int)V;
    ci.off = 4096;
    for (long s = 0; s < V; s++) {
        Site st;
        decode(ci, (int)s, st);
        long r = s;
        int x[4];
        for (int d = 0; d < 3; d++) {
            x[d] = (int)(r % L[d]);
            r /= L[d];
        }
        x[3] = (int)r;
        if (st.g != ci.off + s || x[0] != st.x[0] || x[1] != st.x[1] || x[2] != st.x[2] || x[3] != st.x[3]) {
            std::printf("decode(%ld) on %dx%dx%dx%d: (%d %d %d %d), expected (%d %d %d %d)\n", s, L0, L1, L2, L3,
                        st.x[0], st.x[1], st.x[2], st.x[3], x[0], x[1], x[2], x[3]);
            return 1;
        }
        for (int d = 0; d < 4; d++)
            for (int k = -2; k <= 2; k++) {
                int y[4] = {x[0], x[1], x[2], x[3]};
                y[d] = ((y[d] + k) % L[d] + L[d]) % L[d];
                const long want = ci.off + y[0] + (long)L[0] * (y[1] + (long)L[1] * (y[2] + (long)L[2] * y[3]));
                const int a = nb(ci, st, d, k), b = nb_sel(ci, st, d, k);
                if (a != want || b != want) {
                    std::printf("neighbour of %ld along %d by %d on %dx%dx%dx%d: nb %d, nb_sel %d, expected %ld\n",
                                s, d, k, L0, L1, L2, L3, a, b, want);
                    return 1;
                }
            }
    }
    return 0;
}

int main() {
    for (unsigned d = 2; d <= 4096; d++)
        if (check_divisor(d)) return 1;
    const unsigned big[] = {65535u, 65536u, 65537u, 1000003u, (1u << 30) + 1u, (1u << 31) - 1u};
    for (unsigned d : big)
        if (check_divisor(d)) return 1;
    const int shapes[][4] = {{2, 2, 2, 2}, {3, 5, 7, 2}, {5, 3, 3, 4}, {4, 4, 4, 8}, {6, 6, 6, 6},
                             {8, 12, 16, 4}, {16, 16, 16, 32}, {24, 24, 24, 24}, {48, 48, 48, 8},
                             {17, 31, 13, 9}, {32, 32, 32, 32}};
    for (const auto& s : shapes)
        if (check_lattice(s[0], s[1], s[2], s[3])) return 1;
    std::printf("ok\n");
    return 0;
}
