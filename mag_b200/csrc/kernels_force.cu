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
// the context's tuner times them on live data and keeps the fastest.  The
// staple, force and chain-rule kernels also exist as direction-split shapes
// (3 or 6 warps per 32-link tile, below), which the tuner times for its report
// and which are selected explicitly (mag_set_kernel_variant).
#include "gauge_ops.cuh"
#include "kernels.h"

namespace magb {

namespace {

constexpr int kForceBlock = kForceBlockSites;

// first site of link block b (the block's 128 sites are consecutive); see DevGeom::tile
__device__ __forceinline__ int block_site(const DevGeom& g, int b) {
    if (!g.tile) return b * kForceBlock;
    const int T = g.tile, r = b / g.gpr, grp = b - r * g.gpr;
    const int tid = r / (T * T), w = r - tid * (T * T);
    const int tpr = g.L2 / T;  // tiles along x2
    const int x2 = (tid % tpr) * T + w % T, x3 = (tid / tpr) * T + w / T;
    return ((x3 * g.L2 + x2) * g.gpr + grp) * kForceBlock;
}

__device__ __forceinline__ bool locate_link(const DevGeom& g, ChainInfo& ci, Site& st, int& mu) {
    mu = blockIdx.x & 3;
    const int gs = block_site(g, blockIdx.x >> 2) + threadIdx.x;
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
    W.store(mu, st.g, mul_su3(U.load(mu, st.g), U.load(mu, nb_sel(ci, st, mu, 1))));
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
    if (st.x[0] % m || st.x[1] % m || st.x[2] % m || x3_lattice(ci, st.x[3]) % m) return;
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

// ------------------------------------------------------------ direction split
// One block per (tile of 32 sites, mu) with NS = 3 or 6 warps: warp w computes,
// for the tile's 32 links, direction nu = i + (i >= mu), i = w % 3, either
// whole (NS = 3) or one half of it (NS = 6: half w / 3 of staple_part_near /
// _ext or stout_chain_upper / _lower_acc).  The parts meet in shared memory and
// are added in warp order.  A thread then holds the temporaries of one
// direction (or half) instead of all three, so more warps fit on an SM at a
// register cap R; the shape (NS, R) is what the tuner picks from, next to the
// one-thread-per-link register-cap variants.
__device__ __forceinline__ bool locate_split(const DevGeom& g, ChainInfo& ci, Site& st, int& mu, int& nu, int& w,
                                             int& lane, int& gs) {
    mu = blockIdx.x & 3;
    w = threadIdx.x >> 5;
    lane = threadIdx.x & 31;
    const int i = w % 3;
    nu = i + (i >= mu ? 1 : 0);
    gs = (blockIdx.x >> 2) * MAG_TILE + lane;
    if (gs >= g.vpad) return false;
    ci = g.chains[g.c2c[gs / MAG_CHUNK]];
    const int s = gs - ci.off;
    if (s >= ci.V) return false;
    decode(ci, s, st);
    return true;
}

// parts in shared memory: real component e of warp w's part for lane l at sm[w * 18 + e][l]
template <typename T>
__device__ __forceinline__ void part_put(T (*sm)[MAG_TILE], int w, int lane, const mat3<T>& a) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
        sm[w * 18 + 2 * k][lane] = a.e[k / 3][k % 3].re;
        sm[w * 18 + 2 * k + 1][lane] = a.e[k / 3][k % 3].im;
    }
}
template <int NS, typename T>
__device__ __forceinline__ T part_sum(const T (*sm)[MAG_TILE], int e, int lane) {
    T v = sm[e][lane];
#pragma unroll
    for (int p = 1; p < NS; p++) v = v + sm[p * 18 + e][lane];
    return v;
}
template <int NS, typename T>
__device__ __forceinline__ cplx<T> part_elem(const T (*sm)[MAG_TILE], int k, int lane) {
    return mk(part_sum<NS>(sm, 2 * k, lane), part_sum<NS>(sm, 2 * k + 1, lane));
}
template <int NS, typename T>
__device__ __forceinline__ mat3<T> part_total(const T (*sm)[MAG_TILE], int lane) {
    mat3<T> m;
#pragma unroll
    for (int k = 0; k < 9; k++) m.e[k / 3][k % 3] = part_elem<NS>(sm, k, lane);
    return m;
}

// The NS warps store the tile's 32 result links together: for FP64 warp w
// writes elements w, w + NS, ... (one 512-byte row each); for FP32 the float4
// pairs w, w + NS, ...  elem(k) gives element k = 3 i + j of the link.
template <int NS, typename T, typename F>
__device__ __forceinline__ void split_store(const LinkPlanes<T>& Z, int mu, int gs, int w, F elem) {
    if constexpr (sizeof(T) == 8) {
        cplx<T>* q = const_cast<cplx<T>*>(Z.at(mu, gs));
        for (int k = w; k < 9; k += NS) q[k * MAG_TILE] = elem(k);
    } else {
        float4* q = const_cast<float4*>(Z.at(mu, gs));
        for (int j = w; j < 5; j += NS) {
            const cplx<T> a = elem(2 * j);
            const cplx<T> b = j < 4 ? elem(2 * j + 1) : mk<T>(0, 0);
            q[j * MAG_TILE] = make_float4(a.re, a.im, b.re, b.im);
        }
    }
}
template <typename T>
__device__ __forceinline__ cplx<T> elem_load(const LinkPlanes<T>& Z, int mu, int gs, int k) {
    if constexpr (sizeof(T) == 8) {
        return Z.at(mu, gs)[k * MAG_TILE];
    } else {
        const float4 v = Z.at(mu, gs)[(k / 2) * MAG_TILE];
        return (k & 1) ? mk(v.z, v.w) : mk(v.x, v.y);
    }
}

template <typename T, bool IWA, int NS>
__device__ __forceinline__ mat3<T> staple_split_part(const LinkPlanes<T>& U, const LinkPlanes<T>& W,
                                                     const ChainInfo& ci, const Site& st, int mu, int nu, int w) {
    if (NS == 3 || !IWA) return staple_part<T, IWA>(U, W, ci, st, mu, nu);
    if (w >= 3) return staple_part_ext<T, IWA>(U, W, ci, st, mu, nu);
    mat3<T> A;
    set_zero(A);
    staple_part_near_acc<T, IWA>(A, U, W, ci, st, mu, nu);
    return A;
}

template <typename T, bool IWA, int NS, int R>
__global__ void __maxnreg__(R) k_staple_dagger_split(DevGeom g, LinkPlanes<T> U, LinkPlanes<T> W, LinkPlanes<T> Z) {
    __shared__ T sm[NS * 18][MAG_TILE];
    ChainInfo ci;
    Site st;
    int mu, nu, w, lane, gs;
    const bool ok = locate_split(g, ci, st, mu, nu, w, lane, gs);
    if (ok) part_put(sm, w, lane, staple_split_part<T, IWA, NS>(U, W, ci, st, mu, nu, w));
    __syncthreads();
    if (!ok) return;
    // Z = A^dag: element (i, j) = conj(A(j, i))
    split_store<NS>(Z, mu, gs, w, [&](int k) { return conj(part_elem<NS>(sm, 3 * (k % 3) + k / 3, lane)); });
}

template <typename T, bool IWA, int NS, int R>
__global__ void __maxnreg__(R) k_force_split(DevGeom g, LinkPlanes<T> U, LinkPlanes<T> W, AlgPlanes<T> F) {
    __shared__ T sm[NS * 18][MAG_TILE];
    ChainInfo ci;
    Site st;
    int mu, nu, w, lane, gs;
    const bool ok = locate_split(g, ci, st, mu, nu, w, lane, gs);
    if (ok) part_put(sm, w, lane, staple_split_part<T, IWA, NS>(U, W, ci, st, mu, nu, w));
    __syncthreads();
    if (!ok || w != 0) return;
    const mat3<T> M = mul_nd(U.load(mu, gs), part_total<NS>(sm, lane));
    F.store(mu, gs, i_times_ta(M, (T)(ci.beta / 3.0)));
}

template <typename T, bool TO_FORCE, int NS, int R>
__global__ void __maxnreg__(R) k_stout_chain_split(DevGeom g, LinkPlanes<T> Ul, AlgPlanes<T> Lam, LinkPlanes<T> Zp,
                                                   LinkPlanes<T> Zout, AlgPlanes<T> F) {
    __shared__ T sm[NS * 18][MAG_TILE];
    ChainInfo ci;
    Site st;
    int mu, nu, w, lane, gs;
    const bool ok = locate_split(g, ci, st, mu, nu, w, lane, gs);
    if (ok) {
        const herm8<T> lx = Lam.load(mu, gs);
        mat3<T> t;
        if (NS == 3 || w < 3) {
            t = stout_chain_upper(Ul, Lam, lx, ci, st, mu, nu);
        } else {
            set_zero(t);
        }
        if (NS == 3 || w >= 3) stout_chain_lower_acc(t, Ul, Lam, lx, ci, st, mu, nu);
        part_put(sm, w, lane, t);
    }
    __syncthreads();
    if (!ok) return;
    const T rho = (T)ci.rho;
    if (TO_FORCE) {
        if (w != 0) return;
        // thin level: F = i beta/3 TA(U Z), Z = Z' e^{iQ} + i rho sum of the parts
        mat3<T> z = Zp.load(mu, gs);
        add_to(z, times_i(part_total<NS>(sm, lane), rho));
        F.store(mu, gs, i_times_ta(mul(Ul.load(mu, gs), z), (T)(ci.beta / 3.0)));
    } else {
        split_store<NS>(Zout, mu, gs, w, [&](int k) {
            const cplx<T> p = part_elem<NS>(sm, k, lane), z = elem_load(Zp, mu, gs, k);
            return mk(z.re - rho * p.im, z.im + rho * p.re);
        });
    }
}

unsigned split_blocks(const DevGeom& g) { return (unsigned)(4 * ((g.vpad + MAG_TILE - 1) / MAG_TILE)); }

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
// direction-split variants 4..8 -> (warps per 32-link tile NS, register cap R):
// (3, 168) (3, 128) (6, 168) (6, 128) (6, 96)
#define MAG_BY_SPLIT_VARIANT(v, LAUNCH) \
    switch (v) {                        \
        case 5: LAUNCH(3, 128); break;  \
        case 6: LAUNCH(6, 168); break;  \
        case 7: LAUNCH(6, 128); break;  \
        case 8: LAUNCH(6, 96); break;   \
        default: LAUNCH(3, 168); break; \
    }

template <typename T>
void launch_double_link(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, cudaStream_t s) {
    k_double_link<T><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W);
}
template <typename T>
void launch_force(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, AlgPlanes<T> F, bool iwasaki, int v,
                  cudaStream_t s) {
    if (v >= kNumRegVariants) {
#define L_(NS, R)                                                                                 \
    if (iwasaki) k_force_split<T, true, NS, R><<<split_blocks(g), 32 * NS, 0, s>>>(g, U, W, F); \
    else k_force_split<T, false, 3, R><<<split_blocks(g), 96, 0, s>>>(g, U, W, F);
        MAG_BY_SPLIT_VARIANT(v, L_)
#undef L_
        return;
    }
#define L_(M)                                                                            \
    if (iwasaki) k_force<T, true, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W, F); \
    else k_force<T, false, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, U, W, F);
    MAG_BY_VARIANT(v, L_)
#undef L_
}
template <typename T>
void launch_staple_dagger(const DevGeom& g, LinkPlanes<T> U, LinkPlanes<T> W, LinkPlanes<T> Z, bool iwasaki, int v,
                          cudaStream_t s) {
    if (v >= kNumRegVariants) {
#define L_(NS, R)                                                                                         \
    if (iwasaki) k_staple_dagger_split<T, true, NS, R><<<split_blocks(g), 32 * NS, 0, s>>>(g, U, W, Z); \
    else k_staple_dagger_split<T, false, 3, R><<<split_blocks(g), 96, 0, s>>>(g, U, W, Z);
        MAG_BY_SPLIT_VARIANT(v, L_)
#undef L_
        return;
    }
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
    if (v >= kNumRegVariants) {
#define L_(NS, R)                                                                                     \
    k_stout_chain_split<T, false, NS, R><<<split_blocks(g), 32 * NS, 0, s>>>(g, Ul, Lam, Zp, Zout,     \
                                                                              AlgPlanes<T>{nullptr, 0});
        MAG_BY_SPLIT_VARIANT(v, L_)
#undef L_
        return;
    }
#define L_(M)                                                \
    k_stout_chain<T, false, M><<<link_blocks(g), kForceBlock, 0, s>>>(g, Ul, Lam, Zp, Zout, \
                                                                      AlgPlanes<T>{nullptr, 0});
    MAG_BY_VARIANT(v, L_)
#undef L_
}
template <typename T>
void launch_stout_chain_force(const DevGeom& g, LinkPlanes<T> Ul, AlgPlanes<T> Lam, LinkPlanes<T> Zp, AlgPlanes<T> F,
                              int v, cudaStream_t s) {
    if (v >= kNumRegVariants) {
#define L_(NS, R)                                                                                 \
    k_stout_chain_split<T, true, NS, R><<<split_blocks(g), 32 * NS, 0, s>>>(g, Ul, Lam, Zp,        \
                                                                             LinkPlanes<T>{nullptr, 0}, F);
        MAG_BY_SPLIT_VARIANT(v, L_)
#undef L_
        return;
    }
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
