// kernels_demon.cu -- the per-link demon microcanonical sweep
// (demon_microcanonical, field-demon.h:25-126).
//
// The reference updates the links one after another in site-index order
// (x0 fastest, mu = 0..3 inner), each update seeing every earlier one, and four
// global demons decide every hit: the sweep is sequential by definition.  One
// CTA walks the links of one chain in that order (independent chains of an
// ensemble run side by side, one CTA each) and parallelises inside a link:
//
//  * window: the 353 distinct links that the 168 staple paths of the four links
//    of a site touch are staged in shared memory, one window per site, with
//    16-byte cp.async copies (32 consecutive pieces per instruction); the window
//    of site s + 1 is staged in four parts while warp 0 runs the hits of site s,
//    so the copies hide behind the hits.  The links of sites s and s - 1, which
//    change after a window was staged, are read from three small site buffers
//    that warp 0 keeps current;
//  * paths: 168 threads multiply out one staple path each from the window (two
//    rows of four products and a reconstructed third row; the three-link
//    plaquette paths are padded with a unit slot so every thread runs the same
//    instructions, and adjoints are formed by selects, not by a second product
//    form);
//  * sums: three lanes per component of each of the four staple sums;
//  * hits: warp 0.  A proposal is an SU(2) subgroup element, so a hit's action
//    change only needs the 2x2 block of v S on the subgroup's rows and columns,
//    and the update only changes two rows of the link.  Lanes 0-3 evaluate the
//    first hit for the four demons, lanes 4-11 the second hit after a rejected
//    and after an accepted first hit, so both decisions follow one evaluation.
#include <stdint.h>

#include <cstring>
#include <initializer_list>
#include <vector>

#include "kernels.h"
#include "rng.cuh"

namespace magb {

namespace {

constexpr int kDemonThreads = 256;
constexpr int kPaths = kDemonPaths;  // 6 + 18 + 72 + 72
constexpr int kSteps = 5;
constexpr size_t kLinkBytes = 144;  // 9 complex doubles
constexpr size_t kDemonDynSmem = (2 * kDemonWindow + kPaths) * kLinkBytes;
enum { RNG_DEMON_SU2 = 4, RNG_DEMON_SUBGROUP = 5 };

__device__ __forceinline__ int wrap(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

__device__ __forceinline__ void cp16(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// the draws of random_su3_from_su2(0.9, rng) (field-matrix.h:36-65) from Philox counters
// (link, sweep, hit): a0 uniform in [0.9, 1), a1..a3 in [-1, 1) scaled to |a| = sqrt(1 - a0^2),
// and the SU(2) subgroup (1,2), (0,2) or (0,1) by a draw % 3
__device__ void su2_draw(unsigned long long seed, uint32_t link, uint32_t sweep, uint32_t hit, double a[4], int& sub) {
    uint32_t c1[4] = {link, sweep, hit, (uint32_t)RNG_DEMON_SU2};
    uint32_t c2[4] = {link, sweep, hit, (uint32_t)RNG_DEMON_SUBGROUP};
    philox4x32_10(c1, (uint32_t)seed, (uint32_t)(seed >> 32));
    philox4x32_10(c2, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double small = 0.9;
    auto u = [](uint32_t v) { return ((double)v + 0.5) * 2.3283064365386963e-10; };
    const double a0 = small + (1.0 - small) * u(c1[0]);
    const double a1 = -1.0 + 2.0 * u(c1[1]), a2 = -1.0 + 2.0 * u(c1[2]), a3 = -1.0 + 2.0 * u(c1[3]);
    const double norm = sqrt((1. - a0 * a0) / (a1 * a1 + a2 * a2 + a3 * a3));
    a[0] = a0;
    a[1] = a1 * norm;
    a[2] = a2 * norm;
    a[3] = a3 * norm;
    sub = (int)(c2[0] % 3u);
}

// the proposal is the unit matrix but for rows / columns i, j:
//   m_ii = a0 + i a3, m_ij = a2 + i a1, m_ji = -a2 + i a1, m_jj = a0 - i a3
struct Su2 {
    int i, j;
    cplx<double> ii, ij, ji, jj;
};
__device__ __forceinline__ Su2 su2_of(double a0, double a1, double a2, double a3, int sub) {
    Su2 m;
    m.i = sub == 0 ? 1 : 0;
    m.j = sub == 2 ? 1 : 2;
    m.ii = mk(a0, a3);
    m.ij = mk(a2, a1);
    m.ji = mk(-a2, a1);
    m.jj = mk(a0, -a3);
    return m;
}
__device__ __forceinline__ cplx<double> pick(const cplx<double>& a, const cplx<double>& b, const cplx<double>& c, int r) {
    return r == 0 ? a : (r == 1 ? b : c);
}
// v <- m v when `apply`: rows i, j change
__device__ __forceinline__ void apply_su2(mat3<double>& v, const Su2& m, bool apply) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const cplx<double> vi = pick(v.e[0][c], v.e[1][c], v.e[2][c], m.i);
        const cplx<double> vj = pick(v.e[0][c], v.e[1][c], v.e[2][c], m.j);
        cplx<double> ni = cmul<false, false>(m.ii, vi);
        cmac<false, false, false>(ni, m.ij, vj);
        cplx<double> nj = cmul<false, false>(m.ji, vi);
        cmac<false, false, false>(nj, m.jj, vj);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (apply && r == m.i) v.e[r][c] = ni;
            if (apply && r == m.j) v.e[r][c] = nj;
        }
    }
}
// one column of v <- m v (the operations of apply_su2 on that column)
__device__ __forceinline__ void apply_su2_col(cplx<double> col[3], const Su2& m, bool apply) {
    const cplx<double> vi = pick(col[0], col[1], col[2], m.i);
    const cplx<double> vj = pick(col[0], col[1], col[2], m.j);
    cplx<double> ni = cmul<false, false>(m.ii, vi);
    cmac<false, false, false>(ni, m.ij, vj);
    cplx<double> nj = cmul<false, false>(m.ji, vi);
    cmac<false, false, false>(nj, m.jj, vj);
#pragma unroll
    for (int r = 0; r < 3; r++) {
        if (apply && r == m.i) col[r] = ni;
        if (apply && r == m.j) col[r] = nj;
    }
}
// ReTr(v S) - ReTr(m v S) (field-demon.h:75-78): only the 2x2 block of X = v S on rows and
// columns i, j enters, the other diagonal elements of m X and X being equal
__device__ __forceinline__ double delta_s(const mat3<double>& v, const mat3<double>& S, const Su2& m) {
    cplx<double> vi[3], vj[3], si[3], sj[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        vi[c] = pick(v.e[0][c], v.e[1][c], v.e[2][c], m.i);
        vj[c] = pick(v.e[0][c], v.e[1][c], v.e[2][c], m.j);
        si[c] = pick(S.e[c][0], S.e[c][1], S.e[c][2], m.i);
        sj[c] = pick(S.e[c][0], S.e[c][1], S.e[c][2], m.j);
    }
    cplx<double> xii = cmul<false, false>(vi[0], si[0]), xij = cmul<false, false>(vi[0], sj[0]);
    cplx<double> xji = cmul<false, false>(vj[0], si[0]), xjj = cmul<false, false>(vj[0], sj[0]);
#pragma unroll
    for (int c = 1; c < 3; c++) {
        cmac<false, false, false>(xii, vi[c], si[c]);
        cmac<false, false, false>(xij, vi[c], sj[c]);
        cmac<false, false, false>(xji, vj[c], si[c]);
        cmac<false, false, false>(xjj, vj[c], sj[c]);
    }
    double d = xii.re + xjj.re;
    d = fma(-m.ii.re, xii.re, d);
    d = fma(m.ii.im, xii.im, d);
    d = fma(-m.ij.re, xji.re, d);
    d = fma(m.ij.im, xji.im, d);
    d = fma(-m.ji.re, xij.re, d);
    d = fma(m.ji.im, xij.im, d);
    d = fma(-m.jj.re, xjj.re, d);
    d = fma(m.jj.im, xjj.im, d);
    return d;
}

// a staged link, or its adjoint (by selects: every lane runs the same product code)
__device__ __forceinline__ mat3<double> load_oriented(const double2* q, bool fwd) {
    mat3<double> m;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const double2 v = q[k];
        m.e[k / 3][k % 3] = mk(v.x, v.y);
    }
    mat3<double> o;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            o.e[r][c].re = fwd ? m.e[r][c].re : m.e[c][r].re;
            o.e[r][c].im = fwd ? m.e[r][c].im : -m.e[c][r].im;
        }
    return o;
}

__global__ void __launch_bounds__(kDemonThreads, 1) k_demon_sweep(const DemonJob* jobs, double2* aos,
                                                                  const DemonTables* tabs, int sweep, double e_max,
                                                                  DemonState* states) {
    const ChainInfo ci = jobs[blockIdx.x].ci;
    double2* U = aos + jobs[blockIdx.x].aos_off;
    const unsigned long long seed = jobs[blockIdx.x].seed;
    DemonState* st = states + blockIdx.x;
    extern __shared__ __align__(16) unsigned char dsm[];
    double2* win = reinterpret_cast<double2*>(dsm);  // [2][kDemonWindow][9]: windows of sites s, s + 1
    double(*prod)[18] = reinterpret_cast<double(*)[18]>(dsm + 2 * kDemonWindow * kLinkBytes);  // [kPaths][18]
    __shared__ __align__(16) double2 sbuf[3][4][9];  // links of sites s - 1, s, s + 1 (index site % 3)
    __shared__ double Ssum[4][18];                   // the four staple sums of the current link
    __shared__ double hin_a[2][2][4];                // proposals of this and the next link
    __shared__ int hin_sub[2][2];
    __shared__ uint8_t redir[2][kDemonWindow];  // 0: window slot; 1 + d: link d of the window's site; 5 + d: of the site before
    __shared__ uint16_t sslot[4][kPaths][kSteps];
    __shared__ uint8_t sfwd[4][kPaths][kSteps];
    __shared__ int spk[kDemonWindow];
    __shared__ int snslot;
    for (int i = threadIdx.x; i < 4 * kPaths * kSteps; i += blockDim.x) {
        (&sslot[0][0][0])[i] = (&tabs->slot[0][0][0])[i];
        (&sfwd[0][0][0])[i] = (&tabs->fwd[0][0][0])[i];
    }
    for (int i = threadIdx.x; i < kDemonWindow; i += blockDim.x) spk[i] = tabs->packed[i];
    if (threadIdx.x == 0) snslot = tabs->nslot;
    const int t = threadIdx.x, lane = t & 31;
    double E[4];
#pragma unroll
    for (int k = 0; k < 4; k++) E[k] = st->E[k];
    long long acc = 0, rej = 0;
    __syncthreads();
    const int ns = snslot;
    const int nsite = ci.V;

    // Stage part `part` (0..3; -1: all) of site s's window into buffer wb with the threads
    // [t0, t0 + nthr) (whole warps): lane k of a round forms the source of slot base + k, the
    // round's 32 slots are then copied as 288 consecutive 16-byte pieces.  Part 0 also stages the
    // site's own four links.  Slots holding a link of site s or of sprev are redirected.
    auto stage_site = [&](int s, int wb, int part, int t0, int nthr, int sprev) {
        int x[4];
        int r = s;
        x[0] = r % ci.L[0]; r /= ci.L[0];
        x[1] = r % ci.L[1]; r /= ci.L[1];
        x[2] = r % ci.L[2]; r /= ci.L[2];
        x[3] = r;
        const int n0 = part < 0 ? 0 : (ns * part) / 4, n1 = part < 0 ? ns : (ns * (part + 1)) / 4;
        const int w = (t - t0) >> 5, nw = nthr >> 5;
        if (part <= 0 && w == 0) {
            cp16(&sbuf[s % 3][0][0] + lane, U + (size_t)s * 36 + lane);
            if (lane < 4) cp16(&sbuf[s % 3][0][0] + 32 + lane, U + (size_t)s * 36 + 32 + lane);
        }
        for (int base = n0 + 32 * w; base < n1; base += 32 * nw) {
            const int n = base + lane;
            long long src = -1;
            if (n < n1) {
                const int pk = spk[n];
                const int d = pk >> 16;
                if (d >= 4) {
                    redir[wb][n] = 0;
                    double2* dst = win + ((size_t)wb * kDemonWindow + n) * 9;
#pragma unroll
                    for (int j = 0; j < 9; j++) dst[j] = make_double2(j == 0 || j == 4 || j == 8 ? 1.0 : 0.0, 0.0);
                } else {
                    const int g = wrap(x[0] + (pk & 15) - 4, ci.L[0]) +
                                  wrap(x[1] + ((pk >> 4) & 15) - 4, ci.L[1]) * ci.stride[1] +
                                  wrap(x[2] + ((pk >> 8) & 15) - 4, ci.L[2]) * ci.stride[2] +
                                  wrap(x[3] + ((pk >> 12) & 15) - 4, ci.L[3]) * ci.stride[3];
                    const int code = g == s ? 1 + d : (g == sprev ? 5 + d : 0);
                    redir[wb][n] = (uint8_t)code;
                    if (!code) src = ((long long)g * 4 + d) * 9;
                }
            }
            double2* dst0 = win + ((size_t)wb * kDemonWindow + base) * 9;
#pragma unroll
            for (int rr = 0; rr < 9; rr++) {
                const int f = rr * 32 + lane;
                const int q = f / 9, j = f - 9 * q;
                const long long a = __shfl_sync(0xffffffffu, src, q);
                if (base + q < n1 && a >= 0) cp16(dst0 + f, U + a + j);
            }
        }
        cp_wait_all();
    };

    stage_site(0, 0, -1, 0, kDemonThreads, -1);
    if (t < 2) {
        double a[4];
        int sub;
        su2_draw(seed, 0u, (uint32_t)sweep, (uint32_t)t, a, sub);
        for (int k = 0; k < 4; k++) hin_a[0][t][k] = a[k];
        hin_sub[0][t] = sub;
    }
    __syncthreads();
    const long nlink = 4L * ci.V;
    for (long l = 0; l < nlink; l++) {
        const int s = (int)(l >> 2), mu = (int)(l & 3);
        const int wb = s & 1, hb = (int)(l & 1);
        const int cs = s % 3, ps = (s + 2) % 3;
        // 1. the 168 path products from the window; the last warp draws the next link's proposals
        if (t < kPaths) {
            const uint16_t* sl = sslot[mu][t];
            const uint8_t* fw = sfwd[mu][t];
            auto src = [&](int i) -> const double2* {
                const int slot = sl[i];
                const int code = redir[wb][slot];
                if (code == 0) return win + ((size_t)wb * kDemonWindow + slot) * 9;
                return &sbuf[code < 5 ? cs : ps][(code - 1) & 3][0];
            };
            mat3<double> m = load_oriented(src(0), fw[0]);
#pragma unroll
            for (int i = 1; i < kSteps; i++) m = mul_2r(m, load_oriented(src(i), fw[i]));
            reconstruct_row2(m);
#pragma unroll
            for (int k = 0; k < 9; k++) {
                prod[t][2 * k] = m.e[k / 3][k % 3].re;
                prod[t][2 * k + 1] = m.e[k / 3][k % 3].im;
            }
        } else if (t >= kDemonThreads - 32 && lane < 2 && l + 1 < nlink) {
            double a[4];
            int sub;
            su2_draw(seed, (uint32_t)(l + 1), (uint32_t)sweep, (uint32_t)lane, a, sub);
#pragma unroll
            for (int k = 0; k < 4; k++) hin_a[hb ^ 1][lane][k] = a[k];
            hin_sub[hb ^ 1][lane] = sub;
        }
        __syncthreads();
        // 2. the four staple sums in path order, three lanes (a third of the paths each) per
        //    component, 30 lanes per warp; plaquette and rectangle sums are daggered
        //    (get_staple_dagger / get_rectangular_dagger), chair and twist are not
        {
            const int g = (t >> 5) * 10 + lane / 3, third = lane % 3;
            double a = 0.0;
            int cat = 0, comp = 0;
            if (lane < 30 && g < 72) {
                cat = g / 18;
                comp = g % 18;
                const int p0 = cat == 0 ? 0 : cat == 1 ? 6 : cat == 2 ? 24 : 96;
                const int n = (cat == 0 ? 6 : cat == 1 ? 18 : 72) / 3;
                const int e = comp >> 1, part = comp & 1;
                const int srcc = cat < 2 ? 2 * ((e % 3) * 3 + e / 3) + part : comp;  // element (j, i) for the dagger
                for (int p = p0 + third * n; p < p0 + (third + 1) * n; p++) a += prod[p][srcc];
            }
            const int base = lane - third;
            const double a1 = __shfl_sync(0xffffffffu, a, (base + 1) & 31);
            const double a2 = __shfl_sync(0xffffffffu, a, (base + 2) & 31);
            if (lane < 30 && g < 72 && third == 0) {
                const double sum = (a + a1) + a2;
                Ssum[cat][comp] = (cat < 2 && (comp & 1)) ? -sum : sum;
            }
        }
        __syncthreads();
        // 3. two hits (warp 0; lane 4G + k: demon k; G = 0 the first hit, G = 1 the second after a
        //    rejected first, G = 2 the second after an accepted first); the other warps stage a
        //    quarter of the next site's window
        if (t < 32) {
            mat3<double> v;
#pragma unroll
            for (int c = 0; c < 9; c++) {
                const double2 q = sbuf[cs][mu][c];
                v.e[c / 3][c % 3] = mk(q.x, q.y);
            }
            const int G = lane < 12 ? lane >> 2 : 0, k = lane & 3;
            mat3<double> S;
#pragma unroll
            for (int c = 0; c < 9; c++) S.e[c / 3][c % 3] = mk(Ssum[k][2 * c], Ssum[k][2 * c + 1]);
            const Su2 m0 = su2_of(hin_a[hb][0][0], hin_a[hb][0][1], hin_a[hb][0][2], hin_a[hb][0][3], hin_sub[hb][0]);
            const Su2 m1 = su2_of(hin_a[hb][1][0], hin_a[hb][1][1], hin_a[hb][1][2], hin_a[hb][1][3], hin_sub[hb][1]);
            mat3<double> vs = v;
            apply_su2(vs, m0, G == 2);
            const double dS = delta_s(vs, S, G == 0 ? m0 : m1);
            double d0[4], d1r[4], d1a[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                d0[q] = __shfl_sync(0xffffffffu, dS, q);
                d1r[q] = __shfl_sync(0xffffffffu, dS, 4 + q);
                d1a[q] = __shfl_sync(0xffffffffu, dS, 8 + q);
            }
            bool ok0 = true;
#pragma unroll
            for (int q = 0; q < 4; q++) ok0 = ok0 && E[q] - d0[q] > -e_max && E[q] - d0[q] < e_max;
            if (ok0) {
#pragma unroll
                for (int q = 0; q < 4; q++) E[q] -= d0[q];
                acc++;
            } else {
                rej++;
            }
            bool ok1 = true;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const double d = ok0 ? d1a[q] : d1r[q];
                ok1 = ok1 && E[q] - d > -e_max && E[q] - d < e_max;
            }
            if (ok1) {
#pragma unroll
                for (int q = 0; q < 4; q++) E[q] -= ok0 ? d1a[q] : d1r[q];
                acc++;
            } else {
                rej++;
            }
            // the updated link, one element per lane 0..8: column c of v through both decisions
            {
                const int e = lane < 9 ? lane : 0, r = e / 3, cc = e % 3;
                cplx<double> col[3];
#pragma unroll
                for (int k = 0; k < 3; k++) col[k] = pick(v.e[k][0], v.e[k][1], v.e[k][2], cc);
                apply_su2_col(col, m0, ok0);
                apply_su2_col(col, m1, ok1);
                const cplx<double> o = pick(col[0], col[1], col[2], r);
                if (lane < 9) {
                    const double2 q = make_double2(o.re, o.im);
                    sbuf[cs][mu][lane] = q;
                    U[((size_t)s * 4 + mu) * 9 + lane] = q;
                }
            }
        } else if (s + 1 < nsite) {
            stage_site(s + 1, wb ^ 1, mu, 32, kDemonThreads - 32, s);
        }
        __syncthreads();
    }
    if (t == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) st->E[k] = E[k];
        st->accept += acc;
        st->reject += rej;
    }
}

// the staple paths of a link in direction mu in the reference's order: plaquette staples
// (field-hmc.h:228-239), rectangles (:142-198), chairs and twists (field-staple.h:27-120);
// 0-3 forward, 4-7 backward, -1 pads the three-link paths
void demon_paths(int8_t out[4][kPaths][kSteps]) {
    for (int mu = 0; mu < 4; mu++) {
        int p = 0;
        auto put = [&](std::initializer_list<int> d) {
            int i = 0;
            for (int v : d) out[mu][p][i++] = (int8_t)v;
            for (; i < kSteps; i++) out[mu][p][i] = -1;
            p++;
        };
        for (int nu = 0; nu < 4; nu++) {
            if (nu == mu) continue;
            put({nu, mu, nu + 4});
            put({nu + 4, mu, nu});
        }
        for (int nu = 0; nu < 4; nu++) {
            if (nu == mu) continue;
            put({nu, mu, mu, nu + 4, mu + 4});
            put({nu + 4, mu, mu, nu, mu + 4});
            put({nu, nu, mu, nu + 4, nu + 4});
            put({nu + 4, nu + 4, mu, nu, nu});
            put({mu + 4, nu, mu, mu, nu + 4});
            put({mu + 4, nu + 4, mu, mu, nu});
        }
        for (int twist = 0; twist < 2; twist++)
            for (int nu = 0; nu < 4; nu++) {
                if (nu == mu) continue;
                for (int la = 0; la < 4; la++) {
                    if (la == nu || la == mu) continue;
                    const int chair[4][4] = {{nu, la, la + 4, nu + 4}, {nu, la + 4, la + 4, nu},
                                             {nu + 4, la, la, nu + 4}, {nu + 4, la + 4, la, nu}};
                    const int tw[4][4] = {{nu, la, nu + 4, la + 4}, {nu, la + 4, nu + 4, la},
                                          {nu + 4, la, nu, la + 4}, {nu + 4, la + 4, nu, la}};
                    for (int b = 0; b < 4; b++)
                        for (int ins = 1; ins < 4; ins++) {
                            const int* base = twist ? tw[b] : chair[b];
                            int d[5], k = 0;
                            for (int i = 0; i < 4; i++) {
                                if (i == ins) d[k++] = mu;
                                d[k++] = base[i];
                            }
                            put({d[0], d[1], d[2], d[3], d[4]});
                        }
                }
            }
    }
}

}  // namespace

bool build_demon_tables(DemonTables* T) {
    std::memset(T, 0, sizeof(*T));
    int8_t paths[4][kPaths][kSteps];
    demon_paths(paths);
    // window slots: the distinct (site offset, direction) pairs over the four directions, plus
    // the unit matrix (direction 4) that pads the three-link paths
    std::vector<int> keys;
    auto slot_of = [&](const int y[4], int d) {
        const int key = ((y[0] + 4) & 15) | (((y[1] + 4) & 15) << 4) | (((y[2] + 4) & 15) << 8) |
                        (((y[3] + 4) & 15) << 12) | (d << 16);
        for (size_t k = 0; k < keys.size(); k++)
            if (keys[k] == key) return (int)k;
        keys.push_back(key);
        return (int)keys.size() - 1;
    };
    for (int mu = 0; mu < 4; mu++)
        for (int p = 0; p < kPaths; p++) {
            int y[4] = {0, 0, 0, 0};
            for (int i = 0; i < kSteps; i++) {
                const int d = paths[mu][p][i];
                int sl;
                if (d < 0) {
                    const int z[4] = {0, 0, 0, 0};
                    sl = slot_of(z, 4);
                    T->fwd[mu][p][i] = 1;
                } else {
                    const int a = d & 3;
                    if (d >= 4) y[a]--;
                    if (y[a] < -2 || y[a] > 2) return false;
                    sl = slot_of(y, a);
                    T->fwd[mu][p][i] = d < 4;
                    if (d < 4) y[a]++;
                }
                if (sl >= kDemonWindow) return false;
                T->slot[mu][p][i] = (uint16_t)sl;
            }
        }
    T->nslot = (int)keys.size();
    for (int k = 0; k < T->nslot; k++) T->packed[k] = keys[k];
    return true;
}

void launch_demon_sweeps(const DemonJob* jobs, int njobs, double* aos, const DemonTables* tabs, int sweep,
                         double e_max, DemonState* states, cudaStream_t s) {
    cudaFuncSetAttribute(k_demon_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDemonDynSmem);
    k_demon_sweep<<<(unsigned)njobs, kDemonThreads, kDemonDynSmem, s>>>(jobs, reinterpret_cast<double2*>(aos), tabs,
                                                                        sweep, e_max, states);
}

}  // namespace magb
