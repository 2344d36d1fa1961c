// kernels_demon.cu -- the per-link demon microcanonical sweep
// (demon_microcanonical, field-demon.h:25-126).
//
// The reference updates the links one after another in site-index order
// (x0 fastest, mu = 0..3 inner), each update seeing every earlier one, and four
// global demons decide every hit: the sweep is sequential by definition.  One
// CTA walks the links in that order; the parallelism is inside a link: its 168
// staple paths (6 plaquette, 18 rectangle, 72 chair, 72 twist) are multiplied
// out by 168 threads at once, 72 threads add them up in path order, and warp 0
// runs the two hits (the four action changes on four lanes).
#include <stdint.h>

#include <initializer_list>

#include "kernels.h"
#include "rng.cuh"

namespace magb {

namespace {

constexpr int kDemonThreads = 256;
constexpr int kPaths = kDemonPaths;  // 6 + 18 + 72 + 72
constexpr int kSteps = 5;
enum { RNG_DEMON_SU2 = 4, RNG_DEMON_SUBGROUP = 5 };

__device__ __forceinline__ int wrap(int v, int L) { return v < 0 ? v + L : (v >= L ? v - L : v); }

// The sweep works on an AoS copy of one chain's links (link (s, mu) = 9 complex at
// ((4 s + mu) * 9)): a thread that follows a path reads whole links, two 128-byte
// lines each, which the neighbouring paths and links reuse from L1.
struct AosLinks {
    double2* p;
    __device__ mat3<double> load(int mu, int s) const {
        const double2* q = p + ((size_t)s * 4 + mu) * 9;
        mat3<double> m;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const double2 v = q[k];
            m.e[k / 3][k % 3] = mk(v.x, v.y);
        }
        return m;
    }
    __device__ void store(int mu, int s, const mat3<double>& m) const {
        double2* q = p + ((size_t)s * 4 + mu) * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) q[k] = make_double2(m.e[k / 3][k % 3].re, m.e[k / 3][k % 3].im);
    }
};

// get_path_ordered_product (field-matrix.h:102-131) of the path dir[0..n) from
// site x: forward steps multiply U_d(y) and move, backward steps move and
// multiply U_d(y)^dag; the first factor is taken as it is (I * U = U exactly).
// All link addresses are formed first so the (up to five) loads are in flight
// together.
__device__ mat3<double> path_product(const AosLinks& U, const ChainInfo& ci, const int x[4], const int8_t* dir,
                                     int n) {
    int y[4] = {x[0], x[1], x[2], x[3]};
    int g[kSteps], a[kSteps];
#pragma unroll
    for (int i = 0; i < kSteps; i++) {
        if (i >= n) break;
        const int d = dir[i];
        a[i] = d & 3;
        if (d >= 4) y[a[i]] = wrap(y[a[i]] - 1, ci.L[a[i]]);
        g[i] = y[0] + y[1] * ci.stride[1] + y[2] * ci.stride[2] + y[3] * ci.stride[3];
        if (d < 4) y[a[i]] = wrap(y[a[i]] + 1, ci.L[a[i]]);
    }
    mat3<double> u[kSteps];
#pragma unroll
    for (int i = 0; i < kSteps; i++)
        if (i < n) u[i] = U.load(a[i], g[i]);
    mat3<double> m = dir[0] < 4 ? u[0] : adj(u[0]);
#pragma unroll
    for (int i = 1; i < kSteps; i++)
        if (i < n) m = dir[i] < 4 ? mul(m, u[i]) : mul_nd(m, u[i]);
    return m;
}

// random_su3_from_su2(0.9, rng) (field-matrix.h:36-65) from Philox counters
// (link, sweep, hit): a0 uniform in [0.9, 1), a1..a3 in [-1, 1) scaled to
// |a| = sqrt(1 - a0^2), in the SU(2) subgroup (1,2), (0,2) or (0,1) by a draw % 3
__device__ mat3<double> random_su3_from_su2(unsigned long long seed, uint32_t link, uint32_t sweep, uint32_t hit) {
    uint32_t c1[4] = {link, sweep, hit, (uint32_t)RNG_DEMON_SU2};
    uint32_t c2[4] = {link, sweep, hit, (uint32_t)RNG_DEMON_SUBGROUP};
    philox4x32_10(c1, (uint32_t)seed, (uint32_t)(seed >> 32));
    philox4x32_10(c2, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double small = 0.9;
    auto u = [](uint32_t v) { return ((double)v + 0.5) * 2.3283064365386963e-10; };
    const double a0 = small + (1.0 - small) * u(c1[0]);
    double a1 = -1.0 + 2.0 * u(c1[1]), a2 = -1.0 + 2.0 * u(c1[2]), a3 = -1.0 + 2.0 * u(c1[3]);
    const double norm = sqrt((1. - a0 * a0) / (a1 * a1 + a2 * a2 + a3 * a3));
    a1 *= norm;
    a2 *= norm;
    a3 *= norm;
    mat3<double> m = unit_mat<double>();
    const uint32_t sub = c2[0] % 3u;
    const int i = sub == 0 ? 1 : 0, j = sub == 2 ? 1 : 2;
    m.e[i][i] = mk(a0, a3);
    m.e[i][j] = mk(a2, a1);
    m.e[j][i] = mk(-a2, a1);
    m.e[j][j] = mk(a0, -a3);
    return m;
}

__global__ void __launch_bounds__(kDemonThreads, 1) k_demon_sweep(ChainInfo ci, AosLinks U,
                                                                  const int8_t* paths, unsigned long long seed,
                                                                  int sweep, double e_max, DemonState* st) {
    __shared__ int8_t sp[4 * kPaths * kSteps];
    __shared__ double prod[kPaths][18];
    __shared__ double part3[3][4][18];  // each staple sum in three partial sums
    __shared__ double rnd[2][18];       // the two proposals of the current link
    for (int i = threadIdx.x; i < 4 * kPaths * kSteps; i += blockDim.x) sp[i] = paths[i];
    const int t = threadIdx.x, lane = t & 31;
    double E[4];
#pragma unroll
    for (int k = 0; k < 4; k++) E[k] = st->E[k];
    long long acc = 0, rej = 0;
    __syncthreads();
    const long nlink = 4L * ci.V;
    for (long l = 0; l < nlink; l++) {
        const int s = (int)(l >> 2), mu = (int)(l & 3);
        int x[4];
        {
            int r = s;
            x[0] = r % ci.L[0]; r /= ci.L[0];
            x[1] = r % ci.L[1]; r /= ci.L[1];
            x[2] = r % ci.L[2]; r /= ci.L[2];
            x[3] = r;
        }
        // 1. the 168 path products of this link; the last warp draws the two proposals
        if (t < kPaths) {
            const mat3<double> m = path_product(U, ci, x, sp + (mu * kPaths + t) * kSteps, t < 6 ? 3 : kSteps);
#pragma unroll
            for (int k = 0; k < 9; k++) {
                prod[t][2 * k] = m.e[k / 3][k % 3].re;
                prod[t][2 * k + 1] = m.e[k / 3][k % 3].im;
            }
        } else if (t >= kDemonThreads - 32 && lane < 2) {
            const mat3<double> m = random_su3_from_su2(seed, (uint32_t)l, (uint32_t)sweep, (uint32_t)lane);
#pragma unroll
            for (int k = 0; k < 9; k++) {
                rnd[lane][2 * k] = m.e[k / 3][k % 3].re;
                rnd[lane][2 * k + 1] = m.e[k / 3][k % 3].im;
            }
        }
        __syncthreads();
        // 2. the four staple sums in three partial sums each (216 threads); plaquette and
        //    rectangle sums are daggered (get_staple_dagger / get_rectangular_dagger), chair
        //    and twist are not
        if (t < 216) {
            const int third = t / 72, cat = (t % 72) / 18, comp = t % 18;
            const int p0 = cat == 0 ? 0 : cat == 1 ? 6 : cat == 2 ? 24 : 96;
            const int n = (cat == 0 ? 6 : cat == 1 ? 18 : 72) / 3;
            const int e = comp >> 1, part = comp & 1;
            const int src = cat < 2 ? 2 * ((e % 3) * 3 + e / 3) + part : comp;  // element (j, i) for the dagger
            double a = 0.0;
            for (int p = p0 + third * n; p < p0 + (third + 1) * n; p++) a += prod[p][src];
            part3[third][cat][comp] = (cat < 2 && part) ? -a : a;
        }
        __syncthreads();
        // 3. two hits (warp 0; lane k < 4 owns the action term k): with X_k = v S_k,
        //    delta_S[k] = -ReTr(m X_k) + ReTr(X_k)  (field-demon.h:75-78, (m v) S_k = m (v S_k))
        if (t < 32) {
            const int g = s;
            mat3<double> v = U.load(mu, g);
            mat3<double> Sk;
            const int kk = lane < 4 ? lane : 0;
#pragma unroll
            for (int c = 0; c < 9; c++)
                Sk.e[c / 3][c % 3] = mk(part3[0][kk][2 * c] + part3[1][kk][2 * c] + part3[2][kk][2 * c],
                                        part3[0][kk][2 * c + 1] + part3[1][kk][2 * c + 1] + part3[2][kk][2 * c + 1]);
            mat3<double> X = mul(v, Sk);
            for (int hit = 0; hit < 2; hit++) {
                mat3<double> m;
#pragma unroll
                for (int c = 0; c < 9; c++) m.e[c / 3][c % 3] = mk(rnd[hit][2 * c], rnd[hit][2 * c + 1]);
                const double dS = -retr_mul(m, X) + retr(X);
                double d[4];
                bool ok = true;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    d[k] = __shfl_sync(0xffffffffu, dS, k);
                    ok = ok && E[k] - d[k] > -e_max && E[k] - d[k] < e_max;
                }
                if (ok) {
                    v = mul(m, v);
                    if (hit == 0) X = mul(m, X);
#pragma unroll
                    for (int k = 0; k < 4; k++) E[k] -= d[k];
                    acc++;
                } else {
                    rej++;
                }
            }
            if (lane == 0) U.store(mu, g, v);
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

}  // namespace

void build_demon_paths(int8_t* out) {
    // per mu: plaquette staples (field-hmc.h:228-239), rectangles (:142-198), chairs and
    // twists (field-staple.h:27-120), each list in the reference's order; -1 pads
    for (int mu = 0; mu < 4; mu++) {
        int8_t* o = out + mu * kPaths * kSteps;
        int p = 0;
        auto put = [&](std::initializer_list<int> d) {
            int i = 0;
            for (int v : d) o[p * kSteps + i++] = (int8_t)v;
            for (; i < kSteps; i++) o[p * kSteps + i] = -1;
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

void launch_demon_sweep(const ChainInfo& ci, double* aos, const int8_t* paths, unsigned long long seed, int sweep,
                        double e_max, DemonState* st, cudaStream_t s) {
    k_demon_sweep<<<1, kDemonThreads, 0, s>>>(ci, AosLinks{reinterpret_cast<double2*>(aos)}, paths, seed, sweep,
                                              e_max, st);
}

}  // namespace magb
