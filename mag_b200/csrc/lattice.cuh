// lattice.cuh -- chains, sites and structure-of-arrays field planes.
//
// Every device field lives in one flat "global site" space that concatenates
// the sites of all chains of a context (a single lattice is a context with one
// chain).  Each chain's range starts on a multiple of MAG_CHUNK sites so that
// one lookup, chunk2chain[g / MAG_CHUNK], maps a global site to its chain for
// any block size that divides MAG_CHUNK.
//
// Plane layout (x0 fastest inside a chain, as qlat's index_from_coordinate):
//   link field   : cplx<T> [4 mu][9 elements][Vpad]   (row-major 3x3)
//   algebra field: T       [4 mu][8 compact  ][Vpad]   (see su3.cuh herm8)
// A warp reads 32 consecutive sites of one plane: a 512-byte (double) or
// 256-byte (float) coalesced transaction per matrix element.
#pragma once

#include <stdint.h>

#include "su3.cuh"

#define MAG_CHUNK 256

namespace magb {

struct ChainInfo {
    int L[4];
    int stride[4];
    int V;       // sites of this chain
    int off;     // first global site
    int mag;     // constraint magnification (0: free)
    int pad;
    double beta, c0, c1, rho;
};

struct Site {
    int s;       // local site index inside the chain
    int g;       // global site index
    int x[4];
};

MAG_HD void decode(const ChainInfo& ci, int s, Site& st) {
    st.s = s;
    st.g = ci.off + s;
    int r = s;
    st.x[0] = r % ci.L[0]; r /= ci.L[0];
    st.x[1] = r % ci.L[1]; r /= ci.L[1];
    st.x[2] = r % ci.L[2]; r /= ci.L[2];
    st.x[3] = r;
}

// global index offset of moving k steps (|k| <= L) along d from coordinate xd
MAG_HD int shift_off(const ChainInfo& ci, int xd, int d, int k) {
    int w = xd + k;
    if (w >= ci.L[d]) w -= ci.L[d];
    else if (w < 0) w += ci.L[d];
    return (w - xd) * ci.stride[d];
}

// global index of x + k1 e_d1 + k2 e_d2 + k3 e_d3 (d1, d2, d3 distinct or k = 0)
MAG_HD int nb(const ChainInfo& ci, const Site& st, int d1, int k1) {
    return st.g + shift_off(ci, st.x[d1], d1, k1);
}
MAG_HD int nb(const ChainInfo& ci, const Site& st, int d1, int k1, int d2, int k2) {
    return st.g + shift_off(ci, st.x[d1], d1, k1) + shift_off(ci, st.x[d2], d2, k2);
}

// is_constrained (field-hmc.h:309-337): 0 free, 1 interior, 10 first, 100 last
MAG_HD int constraint_case(const ChainInfo& ci, const Site& st, int mu) {
    const int m = ci.mag;
    if (!m) return 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (i == mu) continue;
        if (st.x[i] % m != 0) return 0;
    }
    const int r = st.x[mu] % m;
    if (r == m - 1) return 100;
    if (r == 0) return 10;
    return 1;
}

template <typename T>
struct LinkPlanes {
    cplx<T>* p;
    long vpad;
    MAG_HD mat3<T> load(int mu, int g) const {
        mat3<T> m;
        const cplx<T>* q = p + (long)mu * 9 * vpad + g;
#pragma unroll
        for (int k = 0; k < 9; k++) m.e[k / 3][k % 3] = q[(long)k * vpad];
        return m;
    }
    MAG_HD void store(int mu, int g, const mat3<T>& m) const {
        cplx<T>* q = p + (long)mu * 9 * vpad + g;
#pragma unroll
        for (int k = 0; k < 9; k++) q[(long)k * vpad] = m.e[k / 3][k % 3];
    }
};

template <typename T>
struct AlgPlanes {
    T* p;
    long vpad;
    MAG_HD herm8<T> load(int mu, int g) const {
        herm8<T> q;
        const T* b = p + (long)mu * 8 * vpad + g;
#pragma unroll
        for (int k = 0; k < 8; k++) q.h[k] = b[(long)k * vpad];
        return q;
    }
    MAG_HD void store(int mu, int g, const herm8<T>& q) const {
        T* b = p + (long)mu * 8 * vpad + g;
#pragma unroll
        for (int k = 0; k < 8; k++) b[(long)k * vpad] = q.h[k];
    }
};

}  // namespace magb
