// lattice.cuh -- chains, sites and structure-of-arrays field planes.
//
// Every device field lives in one flat "global site" space that concatenates
// the sites of all chains of a context (a single lattice is a context with one
// chain).  Each chain's range starts on a multiple of MAG_CHUNK sites so that
// one lookup, chunk2chain[g / MAG_CHUNK], maps a global site to its chain for
// any block size that divides MAG_CHUNK.
//
// Field layout (x0 fastest inside a chain, as qlat's index_from_coordinate):
//   link field   : cplx<T> [4 mu][Vpad / 32 tiles][9 elements][32 sites]
//   algebra field: T       [4 mu][Vpad / 32 tiles][8 compact ][32 sites]
// A warp reads 32 consecutive sites of one element: a 512-byte (double) or
// 256-byte (float) coalesced transaction per matrix element.
#pragma once

#include <stdint.h>
#include <vector_functions.h>
#include <vector_types.h>

#include "su3.cuh"

#define MAG_CHUNK 256

namespace magb {

struct ChainInfo {
    int L[4];
    int stride[4];
    int V;       // sites of this chain
    int off;     // first global site
    int mag;     // constraint magnification (0: free)
    // A shard of a lattice decomposed along x3 holds local x3 in [0, L[3]):
    // the interior [lo3, hi3) and halo slabs on both sides.  Local x3 = 0 is
    // lattice coordinate org3 (mod L3g); Vg counts the whole lattice's sites.
    // An undivided chain has org3 = 0, L3g = L[3], lo3 = 0, hi3 = L[3], Vg = V.
    int org3, L3g, lo3, hi3;
    int Vg;
    // divisors of the site decode: x_d = s / (L_0 ... L_{d-1}) mod L_d without a
    // divide instruction (set_divisors)
    unsigned dm[3];
    int ds[3];
    double beta, c0, c1, rho;
};

// Unsigned division by an invariant d >= 2 (Granlund and Montgomery, "Division
// by invariant integers using multiplication", 1994): with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, which fits 32 bits because 2^l - d < d,
//   n / d = (t + ((n - t) >> 1)) >> (l - 1),  t = floor(n m / 2^32),
// exact for every 32-bit n.
MAG_HD void set_divisor(unsigned d, unsigned& m, int& sh) {
    int l = 0;
    while (l < 32 && (1ull << l) < d) l++;
    m = (unsigned)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
    sh = l - 1;
}
MAG_HD unsigned div_by(unsigned n, unsigned m, int sh) {
#if defined(__CUDA_ARCH__)
    const unsigned t = __umulhi(n, m);
#else
    const unsigned t = (unsigned)(((unsigned long long)n * m) >> 32);
#endif
    return (t + ((n - t) >> 1)) >> sh;
}
// the decode divisors of a chain whose extents L[0..2] are set (each >= 2)
MAG_HD void set_divisors(ChainInfo& ci) {
    for (int d = 0; d < 3; d++) set_divisor((unsigned)ci.L[d], ci.dm[d], ci.ds[d]);
}

struct Site {
    int s;       // local site index inside the chain
    int g;       // global site index
    int x[4];
};

MAG_HD void decode(const ChainInfo& ci, int s, Site& st) {
    st.s = s;
    st.g = ci.off + s;
    unsigned r = (unsigned)s;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const unsigned q = div_by(r, ci.dm[d], ci.ds[d]);
        st.x[d] = (int)(r - q * (unsigned)ci.L[d]);
        r = q;
    }
    st.x[3] = (int)r;
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

// a[d] for a direction d known only at run time, by selects.  Indexing the
// arrays of ChainInfo and Site with a run-time d (as shift_off and nb do)
// places both structs in local memory, so each neighbour address starts with
// L1 loads.  In the staple, force and chain-rule kernels that measured faster
// than selects (fewer registers); in the link update selects measured faster,
// so it takes its neighbour from nb_sel.
MAG_HD int at4(const int (&a)[4], int d) { return d == 0 ? a[0] : d == 1 ? a[1] : d == 2 ? a[2] : a[3]; }
MAG_HD int nb_sel(const ChainInfo& ci, const Site& st, int d, int k) {
    const int L = at4(ci.L, d), xd = at4(st.x, d);
    int w = xd + k;
    if (w >= L) w -= L;
    else if (w < 0) w += L;
    return st.g + (w - xd) * at4(ci.stride, d);
}

// lattice coordinate x3 of local x3 (a shard's halo and interior), and
// whether a site belongs to the chain's own (interior) sites
MAG_HD int x3_lattice(const ChainInfo& ci, int x3) {
    int w = (x3 + ci.org3) % ci.L3g;
    return w < 0 ? w + ci.L3g : w;
}
MAG_HD bool interior(const ChainInfo& ci, const Site& st) { return st.x[3] >= ci.lo3 && st.x[3] < ci.hi3; }
// site index in the whole lattice (x0 fastest); the local index for an undivided chain
MAG_HD long lattice_site(const ChainInfo& ci, const Site& st) {
    return st.x[0] + (long)ci.L[0] * (st.x[1] + (long)ci.L[1] * (st.x[2] + (long)ci.L[2] * x3_lattice(ci, st.x[3])));
}

// is_constrained (field-hmc.h:309-337): 0 free, 1 interior, 10 first, 100 last
// (lattice coordinates, so that a shard classifies its halo as the lattice does)
MAG_HD int constraint_case(const ChainInfo& ci, const Site& st, int mu) {
    const int m = ci.mag;
    if (!m) return 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (i == mu) continue;
        const int xi = i == 3 ? x3_lattice(ci, st.x[3]) : st.x[i];
        if (xi % m != 0) return 0;
    }
    const int r = (mu == 3 ? x3_lattice(ci, st.x[3]) : at4(st.x, mu)) % m;
    if (r == m - 1) return 100;
    if (r == 0) return 10;
    return 1;
}

// Inside one direction the sites are grouped in tiles of MAG_TILE consecutive
// sites; a tile stores element 0 of its MAG_TILE links, then element 1, ...
// (array-of-structure-of-arrays).  A warp of 32 consecutive sites still reads
// one contiguous segment per element, and the elements of one link sit at
// fixed offsets k * MAG_TILE from the first: one address per link, the rest
// are immediate offsets.
#define MAG_TILE 32

template <typename T>
struct LinkPlanes {
    static constexpr int kElems = 9;  // complex slots per link
    cplx<T>* p;
    long vpad;
    MAG_HD const cplx<T>* at(int mu, int g) const {
        return p + (long)mu * 9 * vpad + (long)(g / MAG_TILE) * (9 * MAG_TILE) + (g % MAG_TILE);
    }
    MAG_HD mat3<T> load(int mu, int g) const {
        mat3<T> m;
        const cplx<T>* q = at(mu, g);
#pragma unroll
        for (int k = 0; k < 9; k++) m.e[k / 3][k % 3] = q[k * MAG_TILE];
        return m;
    }
    // rows 0, 1 only (the left factor of a two-row product)
    MAG_HD mat3<T> load_rows01(int mu, int g) const {
        mat3<T> m;
        const cplx<T>* q = at(mu, g);
#pragma unroll
        for (int k = 0; k < 6; k++) m.e[k / 3][k % 3] = q[k * MAG_TILE];
        return m;
    }
    // columns 0, 1 only (the left factor U^dag of a two-row product)
    MAG_HD mat3<T> load_cols01(int mu, int g) const {
        mat3<T> m;
        const cplx<T>* q = at(mu, g);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            m.e[r][0] = q[(3 * r) * MAG_TILE];
            m.e[r][1] = q[(3 * r + 1) * MAG_TILE];
        }
        return m;
    }
    MAG_HD void store(int mu, int g, const mat3<T>& m) const {
        cplx<T>* q = const_cast<cplx<T>*>(at(mu, g));
#pragma unroll
        for (int k = 0; k < 9; k++) q[k * MAG_TILE] = m.e[k / 3][k % 3];
    }
};

// FP32 links: the nine complex elements travel in five 16-byte pairs
// (0,1) (2,3) (4,5) (6,7) (8,-), so a link is five 128-bit loads instead of
// nine 64-bit ones; same tile layout with pairs in place of elements.
template <>
struct LinkPlanes<float> {
    static constexpr int kElems = 10;  // complex slots per link (one padding slot)
    cplx<float>* p;
    long vpad;
    MAG_HD const float4* at(int mu, int g) const {
        return reinterpret_cast<const float4*>(p) + (long)mu * 5 * vpad + (long)(g / MAG_TILE) * (5 * MAG_TILE) +
               (g % MAG_TILE);
    }
    MAG_HD static void put(mat3<float>& m, int k, float re, float im) { m.e[k / 3][k % 3] = mk(re, im); }
    MAG_HD mat3<float> load(int mu, int g) const {
        mat3<float> m;
        const float4* q = at(mu, g);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float4 v = q[j * MAG_TILE];
            put(m, 2 * j, v.x, v.y);
            put(m, 2 * j + 1, v.z, v.w);
        }
        const float4 v = q[4 * MAG_TILE];
        put(m, 8, v.x, v.y);
        return m;
    }
    MAG_HD mat3<float> load_rows01(int mu, int g) const {
        mat3<float> m;
        const float4* q = at(mu, g);
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const float4 v = q[j * MAG_TILE];
            put(m, 2 * j, v.x, v.y);
            put(m, 2 * j + 1, v.z, v.w);
        }
        return m;
    }
    MAG_HD mat3<float> load_cols01(int mu, int g) const {
        mat3<float> m;
        const float4* q = at(mu, g);
        const float4 a = q[0], b = q[MAG_TILE], c = q[2 * MAG_TILE], d = q[3 * MAG_TILE];
        put(m, 0, a.x, a.y);
        put(m, 1, a.z, a.w);
        put(m, 3, b.z, b.w);
        put(m, 4, c.x, c.y);
        put(m, 6, d.x, d.y);
        put(m, 7, d.z, d.w);
        return m;
    }
    MAG_HD void store(int mu, int g, const mat3<float>& m) const {
        float4* q = const_cast<float4*>(at(mu, g));
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const cplx<float> a = m.e[(2 * j) / 3][(2 * j) % 3], b = m.e[(2 * j + 1) / 3][(2 * j + 1) % 3];
            q[j * MAG_TILE] = make_float4(a.re, a.im, b.re, b.im);
        }
        q[4 * MAG_TILE] = make_float4(m.e[2][2].re, m.e[2][2].im, 0.f, 0.f);
    }
};

template <typename T>
struct AlgPlanes {
    T* p;
    long vpad;
    MAG_HD const T* at(int mu, int g) const {
        return p + (long)mu * 8 * vpad + (long)(g / MAG_TILE) * (8 * MAG_TILE) + (g % MAG_TILE);
    }
    MAG_HD herm8<T> load(int mu, int g) const {
        herm8<T> q;
        const T* b = at(mu, g);
#pragma unroll
        for (int k = 0; k < 8; k++) q.h[k] = b[k * MAG_TILE];
        return q;
    }
    MAG_HD void store(int mu, int g, const herm8<T>& q) const {
        T* b = const_cast<T*>(at(mu, g));
#pragma unroll
        for (int k = 0; k < 8; k++) b[k * MAG_TILE] = q.h[k];
    }
};

}  // namespace magb
