// kernels_force.cu -- staple, gauge-force and stout-smearing kernels (sm_100a).
//
// One thread per link.  Blocks are ordered direction-fastest: block b covers
// sites (b / 4) * 128 ... + 127 for mu = b % 4, so the four links of a site
// range are processed at the same time and their shared neighbour links are
// still in L2.  A warp covers 32 consecutive sites of one direction, runs one
// path table and issues coalesced plane loads.  These kernels are bound by the
// CUDA-core FP pipe (3x3 complex products are not a dense contraction; tensor
// cores do not apply).
//
// Every kernel exists in register-cap variants (__launch_bounds__ minimum
// blocks per SM 2, 3, 4, 5 -> at most 255, 168, 128, 102 registers per thread);
// the context's tuner times them on live data and keeps the fastest.
#include "gauge_ops.cuh"
#include "kernels.h"

namespace magb {

namespace {

constexpr int kForceBlock = 128;

__device__ __forceinline__ bool locate_link(const DevGeom& g, ChainInfo& ci, Site& st, int& mu) {
    mu = blockIdx.x & 3;
    const int gs = (blockIdx.x >> 2) * kForceBlock + threadIdx.x;
    if (gs >= g.vpad) return false;
    ci = g.chains[g.c2c[gs / MAG_CHUNK]];
    const int s = gs - ci.off;
    if (s >= ci.V) return false;
    decode(ci, s, st);
    return true;
}

// W(x,mu) = U(x,mu) U(x+mu,mu): the double links of the 1x2 rectangles
template <typename T>
__global__ void __launch_bounds__(kForceBlock) k_double_link(DevGeom g, LinkPlanes<T> U, LinkPlanes<T> W) {
    ChainInfo ci;
    Site st;
    int mu;
    if (!locate_link(g, ci, st, mu)) return;
    W.store(mu, st.g, mul_su3(U.load(mu, st.g), U.load(mu, nb(ci, st, mu, 1))));
}

// F(x,mu) = i beta/3 TA(U(x,mu) A^dag)   (field-hmc.h:394-421, free-link case)
template <typename T, bool IWA, int MINB>
__global__ void __launch_bounds__(kForceBlock, MINB) k_force(DevGeom g, LinkPlanes<T> U, LinkPlanes<T> W,
                                                           AlgPlanes<T> F) {
    ChainInfo ci;
    Site st;
    int mu;
    if (!locate_link(g, ci, st, mu)) return;
    const mat3<T> A = staple_sum<T, IWA>(U, W, ci, st, mu);
    const mat3<T> M = mul_nd(U.load(mu, st.g), A);
    F.store(mu, st.g, i_times_ta(M, (T)(ci.beta / 3.0)));
}

// Z(x,mu) = A^dag  (get_extended_staple_dagger, field-hmc.h:262-269)
template <typename T, bool IWA, int MINB>
__global__ void __launch_bounds__(kForceBlock, MINB) k_staple_dagger(DevGeom g, LinkPlanes<T> U, LinkPlanes<T> W,
                                                                   LinkPlanes<T> Z) {
    ChainInfo ci;
    Site st;
    int mu;
    if (!locate_link(g, ci, st, mu)) return;
    Z.store(mu, st.g, adj(staple_sum<T, IWA>(U, W, ci, st, mu)));
}

// Constrained segments (field-hmc.h:399-407): for a segment of `mag` links
// starting at a coarse site, F_j <- F(x_{j+1}) - U(x_j)^dag F(x_j) U(x_j) for
// j < mag-1 and F_{mag-1} <- 0, from the free-link forces of all its links.
// One thread per coarse site handles the four directions.
template <typename T>
__global__ void k_constraint_fixup(DevGeom g, LinkPlanes<T> U, AlgPlanes<T> F) {
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (gs >= g.vpad) return;
    const ChainInfo ci = g.chains[g.c2c[gs / MAG_CHUNK]];
    const int s = gs - ci.off;
    if (s >= ci.V) return;
    Site st;
    decode(ci, s, st);
    const int m = ci.mag;
    if (!m) return;
    if (st.x[0] % m || st.x[1] % m || st.x[2] % m || st.x[3] % m) return;
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
        int gj = st.g;
        int xj = st.x[mu];
        herm8<T> fj = F.load(mu, gj);
#pragma unroll 1
        for (int j = 0; j < m - 1; j++) {
            const int gn = gj + shift_off(ci, xj, mu, 1);
            const herm8<T> fn = F.load(mu, gn);
            const mat3<T> u = U.load(mu, gj);
            const mat3<T> c = mul(mul_dn(u, expand(fj)), u);  // U^dag F U
            const mat3<T> f = expand(fn);
            herm8<T> out;
            out.h[0] = f.e[0][0].re - c.e[0][0].re;
            out.h[1] = f.e[1][1].re - c.e[1][1].re;
            out.h[2] = f.e[0][1].re - c.e[0][1].re;
            out.h[3] = f.e[0][1].im - c.e[0][1].im;
            out.h[4] = f.e[0][2].re - c.e[0][2].re;
            out.h[5] = f.e[0][2].im - c.e[0][2].im;
            out.h[6] = f.e[1][2].re - c.e[1][2].re;
            out.h[7] = f.e[1][2].im - c.e[1][2].im;
            F.store(mu, gj, out);
            fj = fn;
            gj = gn;
            xj = xj + 1 < ci.L[mu] ? xj + 1 : 0;
        }
        F.store(mu, gj, herm_zero<T>());
    }
}

// One stout level: Q = -i rho TA(stp U^dag) (field-multi.h:32-39), U' = e^{iQ} U
template <typename T, int MINB>
__global__ void __launch_bounds__(kForceBlock, MINB) k_stout_forward(DevGeom g, LinkPlanes<T> Uin,
                                                                   LinkPlanes<T> Uout, AlgPlanes<T> Q) {
    ChainInfo ci;
    Site st;
    int mu;
    if (!locate_link(g, ci, st, mu)) return;
    const mat3<T> stp = plaq_staple_sum(Uin, ci, st, mu);
    const mat3<T> u = Uin.load(mu, st.g);
    const herm8<T> q = i_times_ta(mul_nd(stp, u), (T)(-ci.rho));
    Q.store(mu, st.g, q);
    Uout.store(mu, st.g, mul(expiQ(q), u));
}

template <typename T, int MINB>
__global__ void __launch_bounds__(kForceBlock, MINB) k_stout_lambda(DevGeom g, LinkPlanes<T> Ul, AlgPlanes<T> Q,
                                                                  LinkPlanes<T> Z, AlgPlanes<T> Lam,
                                                                  LinkPlanes<T> Zp) {
    ChainInfo ci;
    Site st;
    int mu;
    if (!locate_link(g, ci, st, mu)) return;
    herm8<T> lam;
    mat3<T> zp;
    stout_lambda(Q.load(mu, st.g), Z.load(mu, st.g), Ul.load(mu, st.g), lam, zp);
    Lam.store(mu, st.g, lam);
    Zp.store(mu, st.g, zp);
}

template <typename T, bool TO_FORCE, int MINB>
__global__ void __launch_bounds__(kForceBlock, MINB) k_stout_chain(DevGeom g, LinkPlanes<T> Ul, AlgPlanes<T> Lam,
                                                                 LinkPlanes<T> Zp, LinkPlanes<T> Zout,
                                                                 AlgPlanes<T> F) {
    ChainInfo ci;
    Site st;
    int mu;
    if (!locate_link(g, ci, st, mu)) return;
    const mat3<T> z = stout_chain(Ul, Lam, Zp, ci, st, mu);
    if (TO_FORCE) {
        // thin level: F = i beta/3 TA(U Z)
        F.store(mu, st.g, i_times_ta(mul(Ul.load(mu, st.g), z), (T)(ci.beta / 3.0)));
    } else {
        Zout.store(mu, st.g, z);
    }
}

unsigned link_blocks(const DevGeom& g) { return (unsigned)(4 * ((g.vpad + kForceBlock - 1) / kForceBlock)); }

}  // namespace

// variant index 0..3 -> minimum blocks per SM 2..5
#define MAG_BY_VARIANT(v, LAUNCH) \
    switch (v) {                  \
        case 1: LAUNCH(3); break; \
        case 2: LAUNCH(4); break; \
        case 3: LAUNCH(5); break; \
        default: LAUNCH(2); break; \
    }

template <typename T>
void launch_double_link(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, cudaStream_t s) {
    k_double_link<T><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W);
}
template <typename T>
void launch_force(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, AlgPlanes<T> F, bool iwasaki, int v,
                  cudaStream_t s) {
#define L_(M)                                                                            \
    if (iwasaki) k_force<T, true, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W, F); \
    else k_force<T, false, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W, F);
    MAG_BY_VARIANT(v, L_)
#undef L_
}
template <typename T>
void launch_staple_dagger(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, LinkPlanes<T> Z, bool iwasaki, int v,
                          cudaStream_t s) {
#define L_(M)                                                                                    \
    if (iwasaki) k_staple_dagger<T, true, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W, Z); \
    else k_staple_dagger<T, false, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W, Z);
    MAG_BY_VARIANT(v, L_)
#undef L_
}
template <typename T>
void launch_constraint_fixup(const DevGeom& g, LinkPlanes<T> U, AlgPlanes<T> F, cudaStream_t s) {
    k_constraint_fixup<T><<<(unsigned)((g.vpad + 255) / 256), 256, 0, s>>>(g, U, F);
}
template <typename T>
void launch_stout_forward(const DevGeom& g, LinkPlanes<T> Uin, LinkPlanes<T> Uout, AlgPlanes<T> Q, int v,
                          cudaStream_t s) {
#define L_(M) k_stout_forward<T, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, Uin, Uout, Q);
    MAG_BY_VARIANT(v, L_)
#undef L_
}
template <typename T>
void launch_stout_lambda(const DevGeom& g, LinkPlanes<T> Ul, AlgPlanes<T> Q, LinkPlanes<T> Z, AlgPlanes<T> Lam,
                         LinkPlanes<T> Zp, int v, cudaStream_t s) {
#define L_(M) k_stout_lambda<T, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, Ul, Q, Z, Lam, Zp);
    MAG_BY_VARIANT(v, L_)
#undef L_
}
template <typename T>
void launch_stout_chain(const DevGeom& g, LinkPlanes<T> Ul, AlgPlanes<T> Lam, LinkPlanes<T> Zp, LinkPlanes<T> Zout,
                        int v, cudaStream_t s) {
#define L_(M)                                                \
    k_stout_chain<T, false, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, Ul, Lam, Zp, Zout, \
                                                                      AlgPlanes<T>{nullptr, 0});
    MAG_BY_VARIANT(v, L_)
#undef L_
}
template <typename T>
void launch_stout_chain_force(const DevGeom& g, LinkPlanes<T> Ul, AlgPlanes<T> Lam, LinkPlanes<T> Zp, AlgPlanes<T> F,
                              int v, cudaStream_t s) {
#define L_(M)                                                                                                   \
    k_stout_chain<T, true, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, Ul, Lam, Zp, LinkPlanes<T>{nullptr, 0}, \
                                                                     F);
    MAG_BY_VARIANT(v, L_)
#undef L_
}

#define MAG_INSTANTIATE(T)                                                                                      \
    template void launch_double_link<T>(const DevGeom&, LinkPlanes<T>, LinkPlanes<T>, cudaStream_t);           \
    template void launch_force<T>(const DevGeom&, LinkPlanes<T>, LinkPlanes<T>, AlgPlanes<T>, bool, int,       \
                                  cudaStream_t);                                                                \
    template void launch_staple_dagger<T>(const DevGeom&, LinkPlanes<T>, LinkPlanes<T>, LinkPlanes<T>, bool,   \
                                          int, cudaStream_t);                                                   \
    template void launch_constraint_fixup<T>(const DevGeom&, LinkPlanes<T>, AlgPlanes<T>, cudaStream_t);       \
    template void launch_stout_forward<T>(const DevGeom&, LinkPlanes<T>, LinkPlanes<T>, AlgPlanes<T>, int,     \
                                          cudaStream_t);                                                        \
    template void launch_stout_lambda<T>(const DevGeom&, LinkPlanes<T>, AlgPlanes<T>, LinkPlanes<T>,          \
                                         AlgPlanes<T>, LinkPlanes<T>, int, cudaStream_t);                      \
    template void launch_stout_chain<T>(const DevGeom&, LinkPlanes<T>, AlgPlanes<T>, LinkPlanes<T>,           \
                                        LinkPlanes<T>, int, cudaStream_t);                                     \
    template void launch_stout_chain_force<T>(const DevGeom&, LinkPlanes<T>, AlgPlanes<T>, LinkPlanes<T>,     \
                                              AlgPlanes<T>, int, cudaStream_t);
MAG_INSTANTIATE(float)
MAG_INSTANTIATE(double)
#undef MAG_INSTANTIATE

}  // namespace magb
