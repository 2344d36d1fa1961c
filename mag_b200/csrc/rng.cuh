// rng.cuh -- counter-based Philox-4x32-10 (Salmon et al., SC'11) streams.
//
// Key = (seed lo, seed hi).  Counters:
//   momenta    (link, block j, trajectory, 1)  -> 8 N(0,1) per link (2 blocks)
//   hot start  (link, block j, 0, 2)           -> 12 N(0,1) per link (3 blocks)
//   accept     (0, 0, trajectory, 3)           -> one 53-bit uniform
// link = 4 * local_site + mu.  Gaussians by Box-Muller on 32-bit uniforms
// (u + 0.5) 2^-32.
#pragma once

#include <stdint.h>

#include "su3.cuh"

namespace magb {

enum { RNG_MOMENTA = 1, RNG_HOT = 2, RNG_ACCEPT = 3 };

MAG_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0; c[1] = (uint32_t)p1; c[2] = n2; c[3] = (uint32_t)p0;
    }
}

MAG_HD void gauss4(unsigned long long seed, uint32_t a, uint32_t b, uint32_t c, uint32_t d, double g[4]) {
    uint32_t ctr[4] = {a, b, c, d};
    philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const double u1 = ((double)ctr[2 * k] + 0.5) * 2.3283064365386963e-10;
        const double u2 = ((double)ctr[2 * k + 1] + 0.5) * 2.3283064365386963e-10;
        const double r = sqrt(-2.0 * log(u1));
        g[2 * k] = r * cos(6.283185307179586 * u2);
        g[2 * k + 1] = r * sin(6.283185307179586 * u2);
    }
}

MAG_HD double uniform53(unsigned long long seed, uint32_t traj) {
    uint32_t ctr[4] = {0u, 0u, traj, (uint32_t)RNG_ACCEPT};
    philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    return ((double)(ctr[0] >> 5) * 67108864.0 + (double)(ctr[1] >> 6)) * (1.0 / 9007199254740992.0);
}

}  // namespace magb
