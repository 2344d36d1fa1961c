// kernels_update.cu -- streaming kernels of the integrator (link updates,
// momentum kicks, reunitarisation), compensated reductions for the
// Hamiltonian, the device-side accept step, RNG and host-layout conversion.
// All of these are bound by HBM bandwidth.
#include "gauge_ops.cuh"
#include "kernels.h"
#include "rng.cuh"

namespace magb {

namespace {

constexpr int kBlock = 256;  // == MAG_CHUNK: a block never spans two chains

__device__ __forceinline__ bool locate(const DevGeom& g, int gs, ChainInfo& ci, Site& st) {
    if (gs >= g.vpad) return false;
    ci = g.chains[g.c2c[gs / MAG_CHUNK]];
    const int s = gs - ci.off;
    if (s >= ci.V) return false;
    decode(ci, s, st);
    return true;
}

unsigned blocks(const DevGeom& g) { return (unsigned)((g.vpad + kBlock - 1) / kBlock); }

// --------------------------------------------------------------- double-double
__device__ __forceinline__ dd2 dd_two_sum(double a, double b) {
    const double s = a + b;
    const double bp = s - a;
    dd2 r;
    r.hi = s;
    r.lo = (a - (s - bp)) + (b - bp);
    return r;
}
__device__ __forceinline__ dd2 dd_add(dd2 a, dd2 b) {
    dd2 s = dd_two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return dd_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dd2 dd_mul(dd2 a, double b) {
    const double p = a.hi * b;
    const double e = fma(a.hi, b, -p);
    return dd_two_sum(p, e + a.lo * b);
}
__device__ __forceinline__ dd2 dd_neg(dd2 a) { a.hi = -a.hi; a.lo = -a.lo; return a; }
__device__ __forceinline__ double dd_val(dd2 a) { return a.hi + a.lo; }

// deterministic block reduction (fixed shuffle tree)
__device__ dd2 block_reduce(dd2 v) {
    __shared__ dd2 sm[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dd2 w;
        w.hi = __shfl_down_sync(0xffffffffu, v.hi, o);
        w.lo = __shfl_down_sync(0xffffffffu, v.lo, o);
        v = dd_add(v, w);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sm[lane] : dd2{0.0, 0.0};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dd2 w;
            w.hi = __shfl_down_sync(0xffffffffu, v.hi, o);
            w.lo = __shfl_down_sync(0xffffffffu, v.lo, o);
            v = dd_add(v, w);
        }
    }
    return v;
}

// ------------------------------------------------------------------- updates
template <typename TU, typename TX>
// two resident blocks per SM (at most 128 registers): a streaming kernel needs the warps
__global__ void __launch_bounds__(kBlock, 2) k_evolve(DevGeom g, LinkPlanes<TU> Uin, LinkPlanes<TU> Uout,
                                                      AlgPlanes<TX> X, double eps,
                         LinkPlanes<float> Ucopy) {
    ChainInfo ci;
    Site st;
    if (!locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st)) return;
    const int mu = blockIdx.y;
    const int cc = constraint_case(ci, st, mu);
    const int gm = nb_sel(ci, st, mu, -1);
    const mat3<TU> r = evolve_link<TU, TX>(Uin.load(mu, st.g), X, eps, cc, st.g, gm, mu);
    Uout.store(mu, st.g, r);
    if (Ucopy.p) Ucopy.store(mu, st.g, convert<float>(r));
}

// P += eps F  (field-hmc.h:427-440)
template <typename TF>
__global__ void k_kick(DevGeom g, AlgPlanes<double> P, AlgPlanes<TF> F, double eps) {
    ChainInfo ci;
    Site st;
    if (!locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st)) return;
    const int mu = blockIdx.y;
    herm8<double> p = P.load(mu, st.g);
    const herm8<TF> f = F.load(mu, st.g);
#pragma unroll
    for (int k = 0; k < 8; k++) p.h[k] += (double)f.h[k] * eps;
    P.store(mu, st.g, p);
}

// reunitarize (field-matrix.h:83-100): CPS Unitarize unless the first two rows
// are exactly zero; the chain's maximum Frobenius deviation is kept.
__global__ void k_reunitarize(DevGeom g, LinkPlanes<double> U, LinkPlanes<float> Ucopy, unsigned long long* reunit) {
    ChainInfo ci;
    Site st;
    double dev = 0.0;
    int chain = -1;
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (locate(g, gs, ci, st)) {
        chain = g.c2c[gs / MAG_CHUNK];
        const int mu = blockIdx.y;
        mat3<double> m = U.load(mu, st.g);
        const mat3<double> old = m;
        bool all_zero = true;
#pragma unroll
        for (int k = 0; k < 6; k++)
            all_zero = all_zero && m.e[k / 3][k % 3].re == 0.0 && m.e[k / 3][k % 3].im == 0.0;
        if (!all_zero) unitarize(m);
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const double dr = m.e[i][j].re - old.e[i][j].re, di = m.e[i][j].im - old.e[i][j].im;
                s += dr * dr + di * di;
            }
        dev = interior(ci, st) ? sqrt(s) : 0.0;  // a shard's halo links are not its own
        U.store(mu, st.g, m);
        if (Ucopy.p) Ucopy.store(mu, st.g, convert<float>(m));
    }
    // block max (all threads of a block belong to one chain or are padding)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dev = fmax(dev, __shfl_down_sync(0xffffffffu, dev, o));
    __shared__ double sm[kBlock / 32];
    __shared__ int chain_sm;
    if (threadIdx.x == 0) chain_sm = -1;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = dev;
    if (chain >= 0) chain_sm = chain;
    __syncthreads();
    if (threadIdx.x == 0 && chain_sm >= 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sm[w]);
        atomicMax(&reunit[chain_sm], (unsigned long long)__double_as_longlong(m));
    }
}

__global__ void k_copy_to_float(DevGeom g, LinkPlanes<double> U, LinkPlanes<float> U32) {
    ChainInfo ci;
    Site st;
    if (!locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st)) return;
    const int mu = blockIdx.y;
    U32.store(mu, st.g, convert<float>(U.load(mu, st.g)));
}

__global__ void k_link_copy(DevGeom g, LinkPlanes<double> src, LinkPlanes<double> dst) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n = g.vpad * 36;
    if (i < n) dst.p[i] = src.p[i];
}

// rejected trajectory: U <- backup for the chain's sites (field-hmc.h:841)
__global__ void k_restore(DevGeom g, LinkPlanes<double> backup, LinkPlanes<double> U, LinkPlanes<float> U32,
                          const ChainState* cs) {
    ChainInfo ci;
    Site st;
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (!locate(g, gs, ci, st)) return;
    if (cs[g.c2c[gs / MAG_CHUNK]].accept) return;
    const int mu = blockIdx.y;
    const mat3<double> m = backup.load(mu, st.g);
    U.store(mu, st.g, m);
    if (U32.p) U32.store(mu, st.g, convert<float>(m));
}

// ---------------------------------------------------------------- reductions
template <typename T>
__global__ void k_action_partials(DevGeom g, LinkPlanes<T> U, int with_rect, dd2* partial) {
    ChainInfo ci;
    Site st;
    dd2 p = {0.0, 0.0}, r = {0.0, 0.0};
    if (locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st) && interior(ci, st)) {
        p.hi = site_plaquette(U, ci, st);
        if (with_rect) r.hi = site_rectangle(U, ci, st);
    }
    p = block_reduce(p);
    r = block_reduce(r);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = p;
        partial[2 * blockIdx.x + 1] = r;
    }
}

// kinetic energy sum of Re Tr(P^2), constrained-last links excluded (field-hmc.h:605-620)
__global__ void k_kinetic_partials(DevGeom g, AlgPlanes<double> P, dd2* partial) {
    ChainInfo ci;
    Site st;
    dd2 k = {0.0, 0.0};
    if (locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st) && interior(ci, st)) {
        double acc = 0.0;
#pragma unroll
        for (int mu = 0; mu < 4; mu++) {
            if (constraint_case(ci, st, mu) == 100) continue;
            acc += retr_sq(P.load(mu, st.g));
        }
        k.hi = acc;
    }
    k = block_reduce(k);
    if (threadIdx.x == 0) partial[2 * blockIdx.x] = k;
}

// per chain: sum the partials of its blocks in block order
// sum over mu of ReTr U(x, mu) (avg_real_trace, field-matrix.h:391-405)
__global__ void k_link_trace_partials(DevGeom g, LinkPlanes<double> U, dd2* partial) {
    ChainInfo ci;
    Site st;
    dd2 k = {0.0, 0.0};
    if (locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st) && interior(ci, st)) {
        double acc = 0.0;
#pragma unroll
        for (int mu = 0; mu < 4; mu++) acc += retr(U.load(mu, st.g));
        k.hi = acc;
    }
    k = block_reduce(k);
    if (threadIdx.x == 0) partial[2 * blockIdx.x] = k;
}
__global__ void k_finalize(DevGeom g, const dd2* partial, int nq, dd2* sums, int slot0, double scale0) {
    const int c = blockIdx.x;
    const ChainInfo ci = g.chains[c];
    const int b0 = ci.off / kBlock, b1 = (ci.off + ci.V + kBlock - 1) / kBlock;
    for (int q = 0; q < nq; q++) {
        dd2 v = {0.0, 0.0};
        for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) v = dd_add(v, partial[2 * b + q]);
        v = block_reduce(v);
        if (threadIdx.x == 0) sums[c * NUM_SLOTS + slot0 + q] = q == 0 ? dd_mul(v, scale0) : v;
        __syncthreads();
    }
}

// ----------------------------------------------------------------- accept
// Metropolis (field-hmc.h:818-843) or trajectory-level demon (field-demon.h:173-186)
__global__ void k_accept(DevGeom g, AcceptArgs a, const dd2* sums, ChainState* cs,
                         const unsigned long long* reunit, TrajRecord* rec, long long* traj_counter) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nchain) return;
    const ChainInfo ci = g.chains[c];
    const long long traj = *traj_counter;
    const dd2* S = sums + c * NUM_SLOTS;
    // S = beta/3 [c0 (-plaq) + c1 (-rect)]  (Wilson: beta/3 (-plaq))
    dd2 pot[2];
    for (int k = 0; k < 2; k++) {
        const dd2 pl = S[k == 0 ? SLOT_PLAQ_OLD : SLOT_PLAQ_NEW];
        const dd2 re = S[k == 0 ? SLOT_RECT_OLD : SLOT_RECT_NEW];
        dd2 t = a.action_iwasaki ? dd_add(dd_mul(dd_neg(pl), ci.c0), dd_mul(dd_neg(re), ci.c1)) : dd_neg(pl);
        pot[k] = dd_mul(t, ci.beta / 3.0);
    }
    const dd2 k0 = S[SLOT_KIN_OLD], k1 = S[SLOT_KIN_NEW];
    const double dh = dd_val(dd_add(dd_add(k1, dd_neg(k0)), dd_add(pot[1], dd_neg(pot[0]))));
    TrajRecord r;
    r.h_old = dd_val(dd_add(k0, pot[0]));
    r.h_new = dd_val(dd_add(k1, pot[1]));
    r.delta_h = dh;
    r.kin_old = dd_val(k0);
    r.kin_new = dd_val(k1);
    r.pot_old = dd_val(pot[0]);
    r.pot_new = dd_val(pot[1]);
    r.plaq_old = dd_val(S[SLOT_PLAQ_OLD]);
    r.plaq_new = dd_val(S[SLOT_PLAQ_NEW]);
    r.rect_old = dd_val(S[SLOT_RECT_OLD]);
    r.rect_new = dd_val(S[SLOT_RECT_NEW]);
    const double u = a.uniform_override ? a.uniform_override[c] : uniform53(a.seed + g.stream_index[c], (uint32_t)traj);
    r.uniform = u;
    ChainState st = cs[c];
    bool acc;
    if (a.metropolis) {
        acc = u < exp(-dh);
        if (traj < a.n_forced) acc = true;
    } else {
        const double ds0 = -dd_val(dd_add(S[SLOT_PLAQ_NEW], dd_neg(S[SLOT_PLAQ_OLD])));
        const double ds1 = -dd_val(dd_add(S[SLOT_RECT_NEW], dd_neg(S[SLOT_RECT_OLD])));
        const double e0 = st.demon0 - ds0, e1 = st.demon1 - ds1;
        acc = e0 > -a.e_max && e0 < a.e_max && e1 > -a.e_max && e1 < a.e_max;
        if (acc) { st.demon0 = e0; st.demon1 = e1; }
    }
    st.accept = acc ? 1 : 0;
    st.naccept += acc ? 1 : 0;
    r.demon0 = st.demon0;
    r.demon1 = st.demon1;
    r.reunit_maxdev = __longlong_as_double((long long)reunit[c]);
    r.avg_plaquette = 0.0;
    r.accept = st.accept;
    r.traj = (int)traj;
    cs[c] = st;
    rec[c] = r;
}

// average thin-link plaquette after accept/reject (field-hmc.h:853-855), then
// advance the trajectory counter
__global__ void k_record_plaquette(DevGeom g, const dd2* sums, TrajRecord* rec, TrajRecord* hist,
                                   const long long* hist_base, int hist_cap, long long* traj_counter) {
    const long long slot = *traj_counter - *hist_base;
    for (int c = threadIdx.x; c < g.nchain; c += blockDim.x) {
        const ChainInfo ci = g.chains[c];
        rec[c].avg_plaquette = dd_val(sums[c * NUM_SLOTS + SLOT_PLAQ_THIN]) / (18.0 * ci.Vg);
        if (hist && slot >= 0 && slot < hist_cap) hist[slot * g.nchain + c] = rec[c];
    }
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) *traj_counter += 1;
}

// --------------------------------------------------------------------- RNG
// P = sum_a T_a xi_a with T_a = lambda_a / sqrt(2) (field-hmc.h:30-69, 681-692)
__global__ void k_momenta(DevGeom g, AlgPlanes<double> P, unsigned long long seed, const long long* traj_counter) {
    ChainInfo ci;
    Site st;
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (!locate(g, gs, ci, st)) return;
    const int mu = blockIdx.y;
    const int chain = g.c2c[gs / MAG_CHUNK];
    const uint32_t link = (uint32_t)(4 * lattice_site(ci, st) + mu);
    const uint32_t traj = (uint32_t)(*traj_counter);
    double xi[8];
    const unsigned long long key = seed + g.stream_index[chain];
    gauss4(key, link, 0u, traj, RNG_MOMENTA, xi);
    gauss4(key, link, 1u, traj, RNG_MOMENTA, xi + 4);
    const double s2 = 1.0 / sqrt(2.0), s6 = 1.0 / sqrt(6.0);
    herm8<double> p;
    p.h[0] = xi[2] * s2 + xi[7] * s6;
    p.h[1] = -xi[2] * s2 + xi[7] * s6;
    p.h[2] = xi[0] * s2;
    p.h[3] = -xi[1] * s2;
    p.h[4] = xi[3] * s2;
    p.h[5] = -xi[4] * s2;
    p.h[6] = xi[5] * s2;
    p.h[7] = -xi[6] * s2;
    P.store(mu, st.g, p);
}

__global__ void k_hot_start(DevGeom g, LinkPlanes<double> U, unsigned long long seed) {
    ChainInfo ci;
    Site st;
    const int gs = blockIdx.x * blockDim.x + threadIdx.x;
    if (!locate(g, gs, ci, st)) return;
    const int mu = blockIdx.y;
    const int chain = g.c2c[gs / MAG_CHUNK];
    const uint32_t link = (uint32_t)(4 * lattice_site(ci, st) + mu);
    double x[12];
    const unsigned long long key = seed + g.stream_index[chain];
    for (int j = 0; j < 3; j++) gauss4(key, link, (uint32_t)j, 0u, RNG_HOT, x + 4 * j);
    mat3<double> m;
    for (int k = 0; k < 3; k++) {
        m.e[0][k] = mk(x[2 * k], x[2 * k + 1]);
        m.e[1][k] = mk(x[6 + 2 * k], x[6 + 2 * k + 1]);
        m.e[2][k] = mk(0.0, 0.0);
    }
    unitarize(m);
    U.store(mu, st.g, m);
}

__global__ void k_cold_start(DevGeom g, LinkPlanes<double> U) {
    ChainInfo ci;
    Site st;
    if (!locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st)) return;
    U.store(blockIdx.y, st.g, unit_mat<double>());
}

// --------------------------------------------------------------- layouts
// host AoS double[V][4][3][3][2] <-> planes
__global__ void k_aos_to_links(const double* aos, int off, int V, LinkPlanes<double> U) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= V) return;
    const int mu = blockIdx.y;
    const double* a = aos + ((long)s * 4 + mu) * 18;
    mat3<double> m;
#pragma unroll
    for (int k = 0; k < 9; k++) m.e[k / 3][k % 3] = mk(a[2 * k], a[2 * k + 1]);
    U.store(mu, off + s, m);
}
template <typename T>
__global__ void k_links_to_aos(LinkPlanes<T> U, int off, int V, double* aos) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= V) return;
    const int mu = blockIdx.y;
    double* a = aos + ((long)s * 4 + mu) * 18;
    const mat3<T> m = U.load(mu, off + s);
#pragma unroll
    for (int k = 0; k < 9; k++) {
        a[2 * k] = (double)m.e[k / 3][k % 3].re;
        a[2 * k + 1] = (double)m.e[k / 3][k % 3].im;
    }
}
template <typename T>
__global__ void k_aos_to_alg(const double* aos, int off, int V, AlgPlanes<T> X) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= V) return;
    const int mu = blockIdx.y;
    const double* a = aos + ((long)s * 4 + mu) * 18;
    herm8<T> q;
    q.h[0] = (T)a[0];
    q.h[1] = (T)a[8];
    q.h[2] = (T)a[2];
    q.h[3] = (T)a[3];
    q.h[4] = (T)a[4];
    q.h[5] = (T)a[5];
    q.h[6] = (T)a[10];
    q.h[7] = (T)a[11];
    X.store(mu, off + s, q);
}
template <typename T>
__global__ void k_alg_to_aos(AlgPlanes<T> X, int off, int V, double* aos) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= V) return;
    const int mu = blockIdx.y;
    double* a = aos + ((long)s * 4 + mu) * 18;
    const mat3<T> m = expand(X.load(mu, off + s));
#pragma unroll
    for (int k = 0; k < 9; k++) {
        a[2 * k] = (double)m.e[k / 3][k % 3].re;
        a[2 * k + 1] = (double)m.e[k / 3][k % 3].im;
    }
}

// CUDA-core FMA throughput probe: eight independent FMA chains per thread
template <typename T>
__global__ void k_fma_probe(T* out, int iters, T b, T c) {
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fma(a[k], b, c);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// packed FP32 probe: eight independent fma.rn.f32x2 chains per thread
__global__ void k_ffma2_probe(float2* out, int iters) {
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = make_float2((float)(threadIdx.x + k) * 1e-3f, (float)k * 1e-3f);
    const float2 b = make_float2(0.999999f, 0.999998f), c = make_float2(1e-6f, 2e-6f);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = __ffma2_rn(a[k], b, c);
    }
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 8; k++) s = __fadd2_rn(s, a[k]);
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// packed FP32 probe with operands formed every iteration from changing pairs:
// i * pair (halves swapped, one negated) and a broadcast half.  Its throughput
// and instruction count next to k_ffma2_probe's show whether such operands
// cost instructions of their own (two packed FMAs per chain and iteration).
__global__ void k_ffma2_sel_probe(float2* out, int iters) {
    float2 a[4], b[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        a[k] = make_float2((float)(threadIdx.x + k) * 1e-3f, (float)k * 1e-3f);
        b[k] = make_float2(0.5f, 0.25f + 1e-3f * k);
    }
    const float2 c = make_float2(1e-6f, 2e-6f);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            a[k] = __ffma2_rn(a[k], make_float2(-b[k].y, b[k].x), c);
            b[k] = __ffma2_rn(b[k], make_float2(a[k].x, a[k].x), c);
        }
    }
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 4; k++) s = __fadd2_rn(s, __fadd2_rn(a[k], b[k]));
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

template <typename T>
void launch_fma_probe(T* out, int nblocks, int iters, cudaStream_t s) {
    k_fma_probe<T><<<nblocks, kBlock, 0, s>>>(out, iters, (T)0.999999, (T)1e-6);
}
void launch_ffma2_probe(void* out, int nblocks, int iters, bool selected_operands, cudaStream_t s) {
    if (selected_operands) k_ffma2_sel_probe<<<nblocks, kBlock, 0, s>>>(static_cast<float2*>(out), iters);
    else k_ffma2_probe<<<nblocks, kBlock, 0, s>>>(static_cast<float2*>(out), iters);
}
template void launch_fma_probe<float>(float*, int, int, cudaStream_t);
template void launch_fma_probe<double>(double*, int, int, cudaStream_t);

template <typename TU, typename TX>
void launch_evolve(const DevGeom& g, LinkPlanes<TU> Uin, LinkPlanes<TU> Uout, AlgPlanes<TX> X, double eps,
                   LinkPlanes<float> Ucopy, cudaStream_t s) {
    k_evolve<TU, TX><<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, Uin, Uout, X, eps, Ucopy);
}
template void launch_evolve<double, double>(const DevGeom&, LinkPlanes<double>, LinkPlanes<double>,
                                            AlgPlanes<double>, double, LinkPlanes<float>, cudaStream_t);
template void launch_evolve<float, float>(const DevGeom&, LinkPlanes<float>, LinkPlanes<float>, AlgPlanes<float>,
                                          double, LinkPlanes<float>, cudaStream_t);
template void launch_evolve<double, float>(const DevGeom&, LinkPlanes<double>, LinkPlanes<double>, AlgPlanes<float>,
                                           double, LinkPlanes<float>, cudaStream_t);

template <typename TF>
void launch_kick(const DevGeom& g, AlgPlanes<double> P, AlgPlanes<TF> F, double eps, cudaStream_t s) {
    k_kick<TF><<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, P, F, eps);
}
template void launch_kick<double>(const DevGeom&, AlgPlanes<double>, AlgPlanes<double>, double, cudaStream_t);
template void launch_kick<float>(const DevGeom&, AlgPlanes<double>, AlgPlanes<float>, double, cudaStream_t);

void launch_reunitarize(const DevGeom& g, LinkPlanes<double> U, LinkPlanes<float> Ucopy,
                        unsigned long long* reunit, cudaStream_t s) {
    k_reunitarize<<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, U, Ucopy, reunit);
}
void launch_copy_to_float(const DevGeom& g, LinkPlanes<double> U, LinkPlanes<float> U32, cudaStream_t s) {
    k_copy_to_float<<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, U, U32);
}
void launch_link_copy(const DevGeom& g, LinkPlanes<double> src, LinkPlanes<double> dst, cudaStream_t s) {
    const long n = g.vpad * 36;
    k_link_copy<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, s>>>(g, src, dst);
}
void launch_restore_rejected(const DevGeom& g, LinkPlanes<double> backup, LinkPlanes<double> U,
                             LinkPlanes<float> U32, const ChainState* st, cudaStream_t s) {
    k_restore<<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, backup, U, U32, st);
}

template <typename T>
void launch_action_sums(const DevGeom& g, LinkPlanes<T> U, bool with_rect, dd2* partial, dd2* sums, int slot_plaq,
                        int slot_rect, cudaStream_t s) {
    k_action_partials<T><<<blocks(g), kBlock, 0, s>>>(g, U, with_rect ? 1 : 0, partial);
    k_finalize<<<g.nchain, kBlock, 0, s>>>(g, partial, 1, sums, slot_plaq, 1.0);
    if (with_rect) k_finalize<<<g.nchain, kBlock, 0, s>>>(g, partial + 1, 1, sums, slot_rect, 1.0);
}
template void launch_action_sums<double>(const DevGeom&, LinkPlanes<double>, bool, dd2*, dd2*, int, int,
                                         cudaStream_t);
template void launch_action_sums<float>(const DevGeom&, LinkPlanes<float>, bool, dd2*, dd2*, int, int,
                                        cudaStream_t);

void launch_link_trace_sum(const DevGeom& g, LinkPlanes<double> U, dd2* partial, dd2* sums, int slot,
                           cudaStream_t s) {
    k_link_trace_partials<<<blocks(g), kBlock, 0, s>>>(g, U, partial);
    k_finalize<<<g.nchain, kBlock, 0, s>>>(g, partial, 1, sums, slot, 1.0);
}
void launch_kinetic_sum(const DevGeom& g, AlgPlanes<double> P, dd2* partial, dd2* sums, int slot, cudaStream_t s) {
    k_kinetic_partials<<<blocks(g), kBlock, 0, s>>>(g, P, partial);
    k_finalize<<<g.nchain, kBlock, 0, s>>>(g, partial, 1, sums, slot, 0.5);
}

void launch_accept(const DevGeom& g, const AcceptArgs& a, dd2* sums, ChainState* st,
                   const unsigned long long* reunit, TrajRecord* rec, long long* traj_counter, cudaStream_t s) {
    k_accept<<<(g.nchain + 63) / 64, 64, 0, s>>>(g, a, sums, st, reunit, rec, traj_counter);
}
void launch_record_plaquette(const DevGeom& g, const dd2* sums, TrajRecord* rec, TrajRecord* hist,
                             const long long* hist_base, int hist_cap, long long* traj_counter, cudaStream_t s) {
    // one block: the counter advances after every chain's record is written
    k_record_plaquette<<<1, 256, 0, s>>>(g, sums, rec, hist, hist_base, hist_cap, traj_counter);
}

void launch_momenta(const DevGeom& g, AlgPlanes<double> P, unsigned long long seed, const long long* traj_counter,
                    cudaStream_t s) {
    k_momenta<<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, P, seed, traj_counter);
}
void launch_hot_start(const DevGeom& g, LinkPlanes<double> U, unsigned long long seed, cudaStream_t s) {
    k_hot_start<<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, U, seed);
}
void launch_cold_start(const DevGeom& g, LinkPlanes<double> U, cudaStream_t s) {
    k_cold_start<<<dim3(blocks(g), 4), kBlock, 0, s>>>(g, U);
}
void launch_aos_to_links(const double* aos, int off, int V, LinkPlanes<double> U, long, cudaStream_t s) {
    k_aos_to_links<<<dim3((V + kBlock - 1) / kBlock, 4), kBlock, 0, s>>>(aos, off, V, U);
}
void launch_links_to_aos(LinkPlanes<double> U, int off, int V, double* aos, cudaStream_t s) {
    k_links_to_aos<double><<<dim3((V + kBlock - 1) / kBlock, 4), kBlock, 0, s>>>(U, off, V, aos);
}
template <typename T>
void launch_links_to_aos_t(LinkPlanes<T> U, int off, int V, double* aos, cudaStream_t s) {
    k_links_to_aos<T><<<dim3((V + kBlock - 1) / kBlock, 4), kBlock, 0, s>>>(U, off, V, aos);
}
template void launch_links_to_aos_t<float>(LinkPlanes<float>, int, int, double*, cudaStream_t);
template void launch_links_to_aos_t<double>(LinkPlanes<double>, int, int, double*, cudaStream_t);
template <typename T>
void launch_aos_to_alg(const double* aos, int off, int V, AlgPlanes<T> X, cudaStream_t s) {
    k_aos_to_alg<T><<<dim3((V + kBlock - 1) / kBlock, 4), kBlock, 0, s>>>(aos, off, V, X);
}
template void launch_aos_to_alg<double>(const double*, int, int, AlgPlanes<double>, cudaStream_t);
template void launch_aos_to_alg<float>(const double*, int, int, AlgPlanes<float>, cudaStream_t);
template <typename T>
void launch_alg_to_aos(AlgPlanes<T> X, int off, int V, double* aos, cudaStream_t s) {
    k_alg_to_aos<T><<<dim3((V + kBlock - 1) / kBlock, 4), kBlock, 0, s>>>(X, off, V, aos);
}
template void launch_alg_to_aos<double>(AlgPlanes<double>, int, int, double*, cudaStream_t);
template void launch_alg_to_aos<float>(AlgPlanes<float>, int, int, double*, cudaStream_t);

}  // namespace magb
