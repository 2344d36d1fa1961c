// kernels_multi.cu -- the two-level coupling of field-multi.h on the GPU (FP64).
//
// A fine field U (the lattice) and a coarse field C (every extent halved) are
// coupled through the stout-smeared blocked links of the fine field:
//   S_eta = -1/eta^2 sum_{coarse x, mu} ReTr(C(x,mu)^dag e^{iQ(2x,mu)} V(2x,mu)),
//   V(y,mu) = U(y,mu) U(y+mu,mu)                 (get_U, field-multi.h:24-27)
//   Q(y,mu) = -i rho TA(stp(y,mu) V(y,mu)^dag)   (get_Q, field-multi.h:29-35)
// with stp the staple of the 2-link (get_staple_rect, field-hmc.h:244-258).
//
// k_multi_coarse: one thread per coarse link; forms V, stp, Q, e^{iQ}, and
// writes the coupling's energy density, the coarse force (get_Cforce,
// field-multi.h:659-683), Lambda = compute_Lambda(Q, C^dag, V) and
// C^dag e^{iQ} (field-multi.h:459-469, the two coarse-link factors the fine
// force needs).
// k_multi_fine: one thread per fine link; adds to the fine gauge force the
// coupling's derivative (get_Fforce, field-multi.h:474-656): by the parity of
// the link's coordinates (stout_type, field-multi.h:378-407) the link is the
// first or second link of a blocked link (types 1, 3: the V term) and lies on
// the 2-link staples of neighbouring coarse links (types 1-4: the paths with
// Lambda inserted, the same path lists as the reference).
#include "gauge_ops.cuh"
#include "kernels.h"

namespace magb {

namespace {

constexpr int kBlock = 128;

// index of lattice coordinate y (any integers; periodic) in a single chain
__device__ __forceinline__ int site_of(const ChainInfo& ci, int y0, int y1, int y2, int y3) {
    auto w = [](int v, int L) {
        v %= L;
        return v < 0 ? v + L : v;
    };
    return ci.off + w(y0, ci.L[0]) + ci.L[0] * (w(y1, ci.L[1]) + ci.L[1] * (w(y2, ci.L[2]) + ci.L[2] * w(y3, ci.L[3])));
}
__device__ __forceinline__ int site_of(const ChainInfo& ci, const int y[4]) { return site_of(ci, y[0], y[1], y[2], y[3]); }

__device__ __forceinline__ mat3<double> link_at(const LinkPlanes<double>& U, const ChainInfo& ci, const int y[4],
                                                int mu) {
    return U.load(mu, site_of(ci, y));
}

// get_path_ordered_product_insertion (field-matrix.h:177-197): directions 0..3
// forward, 4..7 backward, -1 the insertion matrix
__device__ mat3<double> path_insertion(const LinkPlanes<double>& U, const ChainInfo& ci, const int x[4],
                                       const int dir[6], const mat3<double>& ins) {
    int y[4] = {x[0], x[1], x[2], x[3]};
    mat3<double> m = unit_mat<double>();
#pragma unroll 1
    for (int i = 0; i < 6; i++) {
        const int d = dir[i];
        if (d == -1) {
            m = mul(m, ins);
        } else if (d < 4) {
            m = mul(m, link_at(U, ci, y, d));
            y[d]++;
        } else {
            y[d - 4]--;
            m = mul_nd(m, link_at(U, ci, y, d - 4));
        }
    }
    return m;
}

// V(y,mu) and the 2-link staple at fine site y (y = 2 x, x a coarse site)
__device__ void blocked(const LinkPlanes<double>& U, const ChainInfo& cf, const int y[4], int mu, mat3<double>& V,
                        mat3<double>& stp) {
    int z[4] = {y[0], y[1], y[2], y[3]};
    z[mu]++;
    V = mul(link_at(U, cf, y, mu), link_at(U, cf, z, mu));
    set_zero(stp);
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        // U_nu(y) U_mu(y+nu) U_mu(y+nu+mu) U_nu^dag(y+2mu)
        int a[4] = {y[0], y[1], y[2], y[3]};
        a[nu]++;
        int b[4] = {a[0], a[1], a[2], a[3]};
        b[mu]++;
        int c[4] = {y[0], y[1], y[2], y[3]};
        c[mu] += 2;
        mat3<double> t = mul(link_at(U, cf, y, nu), link_at(U, cf, a, mu));
        t = mul(t, link_at(U, cf, b, mu));
        add_to(stp, mul_nd(t, link_at(U, cf, c, nu)));
        // U_nu^dag(y-nu) U_mu(y-nu) U_mu(y-nu+mu) U_nu(y-nu+2mu)
        int d[4] = {y[0], y[1], y[2], y[3]};
        d[nu]--;
        int e[4] = {d[0], d[1], d[2], d[3]};
        e[mu]++;
        int f[4] = {d[0], d[1], d[2], d[3]};
        f[mu] += 2;
        t = mul_dn(link_at(U, cf, d, nu), link_at(U, cf, d, mu));
        t = mul(t, link_at(U, cf, e, mu));
        add_to(stp, mul(t, link_at(U, cf, f, nu)));
    }
}

__device__ __forceinline__ dd2 m_two_sum(double a, double b) {
    const double s = a + b, bp = s - a;
    return dd2{s, (a - (s - bp)) + (b - bp)};
}
__device__ __forceinline__ dd2 m_add(dd2 a, dd2 b) {
    dd2 s = m_two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return m_two_sum(s.hi, s.lo);
}
__device__ dd2 m_block_reduce(dd2 v) {
    __shared__ dd2 sm[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dd2 w{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
        v = m_add(v, w);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sm[lane] : dd2{0.0, 0.0};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dd2 w{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
            v = m_add(v, w);
        }
    }
    return v;
}

// grid: (coarse sites / kBlock) x 4 directions
__global__ void k_multi_coarse(ChainInfo cf, ChainInfo cc, LinkPlanes<double> U, LinkPlanes<double> C,
                               double rho, double eta_sqr, AlgPlanes<double> Fc, AlgPlanes<double> Lam,
                               LinkPlanes<double> Zp, dd2* partial) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int mu = blockIdx.y;
    dd2 e{0.0, 0.0};
    if (s < cc.V) {
        Site st;
        decode(cc, s, st);
        const int y[4] = {2 * st.x[0], 2 * st.x[1], 2 * st.x[2], 2 * st.x[3]};
        mat3<double> V, stp;
        blocked(U, cf, y, mu, V, stp);
        const herm8<double> q = i_times_ta(mul_nd(stp, V), -rho);
        const mat3<double> G = mul(expiQ(q), V);
        const mat3<double> c = C.load(mu, st.g);
        e.hi = retr_mul_nd(G, c);  // ReTr(C^dag G) = ReTr(G C^dag)
        if (Fc.p) Fc.store(mu, st.g, i_times_ta(mul_nd(c, G), 1.0 / eta_sqr));
        if (Lam.p) {
            herm8<double> lam;
            mat3<double> zp;
            stout_lambda(q, adj(c), V, lam, zp);  // compute_Lambda(Q, C^dag, V) and C^dag e^{iQ}
            Lam.store(mu, st.g, lam);
            Zp.store(mu, st.g, zp);
        }
    }
    if (partial) {
        e = m_block_reduce(e);
        if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = e;
    }
}

// sum of the partials in a fixed order (one block)
__global__ void k_multi_sum(const dd2* partial, int n, dd2* out) {
    dd2 v{0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) v = m_add(v, partial[i]);
    v = m_block_reduce(v);
    if (threadIdx.x == 0) *out = v;
}

// F(x,mu) += i/eta^2 TA(U(x,mu) T(x,mu)), T the coupling's derivative terms (get_Fforce)
__global__ void k_multi_fine(ChainInfo cf, ChainInfo cc, LinkPlanes<double> U, AlgPlanes<double> Lam,
                             LinkPlanes<double> Zp, double rho, double eta_sqr, AlgPlanes<double> F) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int mu = blockIdx.y;
    if (s >= cf.V) return;
    Site st;
    decode(cf, s, st);
    const int* x = st.x;
    // stout_type
    int odd[4], n = 0;
#pragma unroll
    for (int i = 0; i < 4; i++)
        if (x[i] & 1) odd[n++] = i;
    int type = 0, o = 0;
    if (n == 0) type = 1;
    else if (n == 1) {
        if (odd[0] == mu) type = 3;
        else { type = 2; o = odd[0]; }
    } else if (n == 2) {
        if (odd[0] == mu) { type = 4; o = odd[1]; }
        else if (odd[1] == mu) { type = 4; o = odd[0]; }
    }
    if (type == 0) return;
    const int sx[4] = {x[0] + (mu == 0), x[1] + (mu == 1), x[2] + (mu == 2), x[3] + (mu == 3)};  // paths start at x + mu
    // coarse-link quantities at fine coordinate y = x + shifts (y even): Lambda, C^dag e^{iQ}
    auto cidx = [&](int d1, int k1, int d2, int k2) {
        int y[4] = {x[0], x[1], x[2], x[3]};
        if (d1 >= 0) y[d1] += k1;
        if (d2 >= 0) y[d2] += k2;
        return site_of(cc, y[0] >> 1, y[1] >> 1, y[2] >> 1, y[3] >> 1);  // y even: exact halves (floor)
    };
    auto lam = [&](int c, int dir) { return expand(Lam.load(dir, c)); };
    mat3<double> t;
    set_zero(t);
    auto ins = [&](int d0, int d1, int d2, int d3, int d4, int d5, const mat3<double>& m, double sgn) {
        const int dir[6] = {d0, d1, d2, d3, d4, d5};
        const mat3<double> p = path_insertion(U, cf, sx, dir, m);
        // t += sgn * i rho * p
        add_to(t, times_i(p, sgn * rho));
    };
    if (type == 1) {
        const int c0 = cidx(-1, 0, -1, 0);
        t = mul(U.load(mu, nb(cf, st, mu, 1)), Zp.load(mu, c0));  // U(x+mu) C^dag e^{iQ}
#pragma unroll 1
        for (int nu = 0; nu < 4; nu++) {
            if (nu == mu) continue;
            const mat3<double> lm = lam(c0, mu), ln = lam(c0, nu);
            ins(mu, nu, mu + 4, mu + 4, nu + 4, -1, lm, 1.0);
            ins(mu, nu + 4, mu + 4, mu + 4, nu, -1, lm, 1.0);
            ins(nu, nu, mu + 4, nu + 4, nu + 4, -1, ln, -1.0);
            ins(nu + 4, nu + 4, mu + 4, -1, nu, nu, lam(cidx(nu, -2, -1, 0), nu), 1.0);
        }
    } else if (type == 2) {
        ins(mu, o + 4, mu + 4, mu + 4, -1, o, lam(cidx(o, -1, -1, 0), mu), -1.0);
        ins(mu, o, mu + 4, mu + 4, -1, o + 4, lam(cidx(o, 1, -1, 0), mu), -1.0);
    } else if (type == 3) {
        const int c0 = cidx(mu, -1, -1, 0);
        t = mul(Zp.load(mu, c0), U.load(mu, nb(cf, st, mu, -1)));  // C^dag e^{iQ} U(x-mu)
#pragma unroll 1
        for (int nu = 0; nu < 4; nu++) {
            if (nu == mu) continue;
            const mat3<double> lm = lam(c0, mu);
            ins(nu, mu + 4, mu + 4, nu + 4, -1, mu, lm, 1.0);
            ins(nu + 4, mu + 4, mu + 4, nu, -1, mu, lm, 1.0);
            ins(-1, nu, nu, mu + 4, nu + 4, nu + 4, lam(cidx(mu, 1, -1, 0), nu), 1.0);
            ins(nu + 4, nu + 4, -1, mu + 4, nu, nu, lam(cidx(mu, 1, nu, -2), nu), -1.0);
        }
    } else {  // type 4
        ins(o + 4, mu + 4, mu + 4, -1, o, mu, lam(cidx(o, -1, mu, -1), mu), -1.0);
        ins(o, mu + 4, mu + 4, -1, o + 4, mu, lam(cidx(o, 1, mu, -1), mu), -1.0);
    }
    const herm8<double> add = i_times_ta(mul(U.load(mu, st.g), t), 1.0 / eta_sqr);
    herm8<double> f = F.load(mu, st.g);
#pragma unroll
    for (int k = 0; k < 8; k++) f.h[k] += add.h[k];
    F.store(mu, st.g, f);
}

}  // namespace

void launch_multi_coarse(const ChainInfo& cf, const ChainInfo& cc, LinkPlanes<double> U, LinkPlanes<double> C,
                         double rho, double eta_sqr, AlgPlanes<double> Fc, AlgPlanes<double> Lam, LinkPlanes<double> Zp,
                         dd2* partial, dd2* energy, cudaStream_t s) {
    const unsigned nb = (unsigned)((cc.V + kBlock - 1) / kBlock);
    k_multi_coarse<<<dim3(nb, 4), kBlock, 0, s>>>(cf, cc, U, C, rho, eta_sqr, Fc, Lam, Zp, partial);
    if (partial && energy) k_multi_sum<<<1, kBlock, 0, s>>>(partial, (int)(4 * nb), energy);
}

void launch_multi_fine(const ChainInfo& cf, const ChainInfo& cc, LinkPlanes<double> U, AlgPlanes<double> Lam,
                       LinkPlanes<double> Zp, double rho, double eta_sqr, AlgPlanes<double> F, cudaStream_t s) {
    const unsigned nb = (unsigned)((cf.V + kBlock - 1) / kBlock);
    k_multi_fine<<<dim3(nb, 4), kBlock, 0, s>>>(cf, cc, U, Lam, Zp, rho, eta_sqr, F);
}

}  // namespace magb
