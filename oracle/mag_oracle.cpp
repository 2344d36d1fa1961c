// mag_oracle.cpp -- FP64 CPU oracle for mag's constrained SU(3) HMC path.
//
// TEST INFRASTRUCTURE ONLY.  Loaded by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker; the product library never links
// or calls it.
//
// PARITY UNPINNED: the reference publishes no golden vectors or known-answer
// tests, and it cannot be compiled here (it needs CPS, Qlattice, QMP, MPI).
// Each function below restates the reference function named in its comment,
// keeping its operation order where the reference fixes one; the tests pin the
// restatement with invariants instead of reference outputs.
//
// Deviations from the reference, all deliberate:
//  * acos(c0/c0max) in expiQ/DexpiQ/compute_Lambda clamps its argument to <= 1
//    (rounding can push it above 1 and the reference then returns NaN).
//  * global sums (action, kinetic energy) are double-double compensated over a
//    per-site array in site order, so they do not depend on the thread count
//    (the reference adds per-thread partials, field-matrix.h:306-329).
//  * momenta, hot starts and Metropolis uniforms come from Philox-4x32-10
//    streams instead of Qlattice's SHA-256 RngState (not reproducible here).
//  * thin-link multi-level stout smearing is the isotropic 4-D generalisation
//    of the reference's blocked single-level stout (field-multi.h:32-39); its
//    derivative chains compute_Lambda (field-multi.h:180-269) through every level.
#include "mag_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

typedef std::complex<double> cplx;

struct M3 {
    double v[18];  // element (r,c): re at v[2*(3r+c)], im at v[2*(3r+c)+1]
};

inline M3 zero3() { M3 m; for (int i = 0; i < 18; i++) m.v[i] = 0.0; return m; }
inline M3 unit3() { M3 m = zero3(); m.v[0] = m.v[8] = m.v[16] = 1.0; return m; }
inline cplx get(const M3& m, int r, int c) { return cplx(m.v[2 * (3 * r + c)], m.v[2 * (3 * r + c) + 1]); }
inline void set(M3& m, int r, int c, cplx z) { m.v[2 * (3 * r + c)] = z.real(); m.v[2 * (3 * r + c) + 1] = z.imag(); }

inline M3 mul(const M3& a, const M3& b) {
    M3 c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double re = 0.0, im = 0.0;
            for (int k = 0; k < 3; k++) {
                const double ar = a.v[2 * (3 * i + k)], ai = a.v[2 * (3 * i + k) + 1];
                const double br = b.v[2 * (3 * k + j)], bi = b.v[2 * (3 * k + j) + 1];
                re += ar * br - ai * bi;
                im += ar * bi + ai * br;
            }
            c.v[2 * (3 * i + j)] = re;
            c.v[2 * (3 * i + j) + 1] = im;
        }
    return c;
}
inline M3 dag(const M3& a) {
    M3 c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            c.v[2 * (3 * i + j)] = a.v[2 * (3 * j + i)];
            c.v[2 * (3 * i + j) + 1] = -a.v[2 * (3 * j + i) + 1];
        }
    return c;
}
inline M3 operator+(const M3& a, const M3& b) { M3 c; for (int i = 0; i < 18; i++) c.v[i] = a.v[i] + b.v[i]; return c; }
inline M3 operator-(const M3& a, const M3& b) { M3 c; for (int i = 0; i < 18; i++) c.v[i] = a.v[i] - b.v[i]; return c; }
inline M3& operator+=(M3& a, const M3& b) { for (int i = 0; i < 18; i++) a.v[i] += b.v[i]; return a; }
inline M3 operator*(const M3& a, double s) { M3 c; for (int i = 0; i < 18; i++) c.v[i] = a.v[i] * s; return c; }
inline M3 operator*(const M3& a, const M3& b) { return mul(a, b); }
inline M3 cscale(const M3& a, cplx z) {
    M3 c;
    for (int i = 0; i < 9; i++) {
        const double ar = a.v[2 * i], ai = a.v[2 * i + 1];
        c.v[2 * i] = ar * z.real() - ai * z.imag();
        c.v[2 * i + 1] = ar * z.imag() + ai * z.real();
    }
    return c;
}
inline double retr(const M3& a) { return a.v[0] + a.v[8] + a.v[16]; }
inline cplx tr(const M3& a) { return cplx(a.v[0] + a.v[8] + a.v[16], a.v[1] + a.v[9] + a.v[17]); }

// cps::Matrix::TrLessAntiHermMatrix: 1/2 (M - M^dag) - 1/6 Tr(M - M^dag)
inline M3 ta(const M3& m) {
    M3 c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            c.v[2 * (3 * i + j)] = 0.5 * (m.v[2 * (3 * i + j)] - m.v[2 * (3 * j + i)]);
            c.v[2 * (3 * i + j) + 1] = 0.5 * (m.v[2 * (3 * i + j) + 1] + m.v[2 * (3 * j + i) + 1]);
        }
    const double t = (c.v[1] + c.v[9] + c.v[17]) / 3.0;
    c.v[1] -= t; c.v[9] -= t; c.v[17] -= t;
    return c;
}

// field-multi.h:41-45 hermitian_traceless
inline M3 hermitian_traceless(const M3& m) {
    const M3 s = m + dag(m);
    const cplx t = tr(s) / 3.0;
    M3 c = s;
    for (int k = 0; k < 3; k++) {
        c.v[8 * k] -= t.real();
        c.v[8 * k + 1] -= t.imag();
    }
    return c * 0.5;
}

// cps::Matrix::Unitarize: Gram-Schmidt on rows 0,1; row 2 = conj(row0 x row1)
inline void unitarize(M3& m) {
    cplx r0[3], r1[3];
    for (int k = 0; k < 3; k++) { r0[k] = get(m, 0, k); r1[k] = get(m, 1, k); }
    double n0 = 0.0;
    for (int k = 0; k < 3; k++) n0 += std::norm(r0[k]);
    n0 = 1.0 / std::sqrt(n0);
    for (int k = 0; k < 3; k++) r0[k] *= n0;
    cplx c(0.0, 0.0);
    for (int k = 0; k < 3; k++) c += std::conj(r0[k]) * r1[k];
    for (int k = 0; k < 3; k++) r1[k] -= c * r0[k];
    double n1 = 0.0;
    for (int k = 0; k < 3; k++) n1 += std::norm(r1[k]);
    n1 = 1.0 / std::sqrt(n1);
    for (int k = 0; k < 3; k++) r1[k] *= n1;
    cplx r2[3];
    r2[0] = std::conj(r0[1] * r1[2] - r0[2] * r1[1]);
    r2[1] = std::conj(r0[2] * r1[0] - r0[0] * r1[2]);
    r2[2] = std::conj(r0[0] * r1[1] - r0[1] * r1[0]);
    for (int k = 0; k < 3; k++) { set(m, 0, k, r0[k]); set(m, 1, k, r1[k]); set(m, 2, k, r2[k]); }
}

// field-matrix.h:75-81 norm (Frobenius)
inline double fnorm(const M3& m) {
    double s = 0.0;
    for (int i = 0; i < 18; i++) s += m.v[i] * m.v[i];
    return std::sqrt(s);
}

inline cplx expix(double x) { return cplx(std::cos(x), std::sin(x)); }
const cplx I(0.0, 1.0);

// Cayley-Hamilton coefficients shared by expiQ, DexpiQ and compute_Lambda
// (field-hmc.h:88-115, field-multi.h:92-168).
struct CH {
    bool trivial;
    bool reflect;
    double u, w, xi0, xi1;
    cplx f0, f1, f2, b10, b11, b12, b20, b21, b22;
};

inline CH ch_coeffs(const M3& Q, bool with_b) {
    CH r;
    r.trivial = false;
    double c0 = retr(Q * Q * Q) / 3.0;
    r.reflect = false;
    if (c0 < 0.0) { c0 = -c0; r.reflect = true; }
    const double c1 = retr(Q * Q) / 2.0;
    if (c1 == 0.0) { r.trivial = true; return r; }
    const double c0m = 2.0 * std::pow(c1 / 3.0, 1.5);
    const double theta = std::acos(std::min(c0 / c0m, 1.0));
    const double u = std::sqrt(c1 / 3.0) * std::cos(theta / 3.0);
    const double w = std::sqrt(c1) * std::sin(theta / 3.0);
    double xi0, xi1;
    if (w * w < 0.05 * 0.05) {
        xi0 = 1. - w * w / 6. * (1. - w * w / 20. * (1. - w * w / 42.));
        xi1 = -1. / 2. * (1. - w * w / 12. * (1. - w * w / 30.)) + 1. / 6. * (1. - w * w / 20. * (1. - w * w / 42.));
    } else {
        xi0 = std::sin(w) / w;
        xi1 = std::cos(w) / (w * w) - std::sin(w) / (w * w * w);
    }
    const cplx e2u = expix(2. * u), emu = expix(-u);
    const double cw = std::cos(w);
    const cplx h0 = (u * u - w * w) * e2u + emu * (8. * u * u * cw + I * 2. * u * (3. * u * u + w * w) * xi0);
    const cplx h1 = 2. * u * e2u - emu * (2. * u * cw - I * (3. * u * u - w * w) * xi0);
    const cplx h2 = e2u - emu * (cw + I * 3. * u * xi0);
    const double den = 9. * u * u - w * w;
    r.f0 = h0 / den; r.f1 = h1 / den; r.f2 = h2 / den;
    r.u = u; r.w = w; r.xi0 = xi0; r.xi1 = xi1;
    if (with_b) {
        const cplx r01 = 2. * (u + I * (u * u - w * w)) * e2u +
                         2. * emu * (4. * u * (2. - I * u) * cw + I * xi0 * (9. * u * u + w * w - I * u * (3. * u * u + w * w)));
        const cplx r11 = 2. * (1. + 2. * I * u) * e2u + emu * (-2. * (1. - I * u) * cw + I * xi0 * (6. * u + I * (w * w - 3. * u * u)));
        const cplx r21 = 2. * I * e2u + I * emu * (cw - 3. * xi0 * (1. - I * u));
        const cplx r02 = -2. * e2u + 2. * I * u * emu * (cw + (1. + 4. * I * u) * xi0 + 3. * u * u * xi1);
        const cplx r12 = -I * emu * (cw + (1. + 2. * I * u) * xi0 - 3. * u * u * xi1);
        const cplx r22 = emu * (xi0 - 3. * I * u * xi1);
        const double bden = 2. * den * den;
        r.b10 = (2. * u * r01 + (3. * u * u - w * w) * r02 - 2. * (15. * u * u + w * w) * r.f0) / bden;
        r.b11 = (2. * u * r11 + (3. * u * u - w * w) * r12 - 2. * (15. * u * u + w * w) * r.f1) / bden;
        r.b12 = (2. * u * r21 + (3. * u * u - w * w) * r22 - 2. * (15. * u * u + w * w) * r.f2) / bden;
        r.b20 = (r01 - 3. * u * r02 - 24. * u * r.f0) / bden;
        r.b21 = (r11 - 3. * u * r12 - 24. * u * r.f1) / bden;
        r.b22 = (r21 - 3. * u * r22 - 24. * u * r.f2) / bden;
    }
    if (r.reflect) {
        r.f0 = std::conj(r.f0); r.f1 = -std::conj(r.f1); r.f2 = std::conj(r.f2);
        if (with_b) {
            r.b10 = std::conj(r.b10); r.b11 = -std::conj(r.b11); r.b12 = std::conj(r.b12);
            r.b20 = -std::conj(r.b20); r.b21 = std::conj(r.b21); r.b22 = -std::conj(r.b22);
        }
    }
    return r;
}

// field-hmc.h:82-123 expiQ
inline M3 expiQ(const M3& Q) {
    CH c = ch_coeffs(Q, false);
    if (c.trivial) return unit3();
    return cscale(unit3(), c.f0) + cscale(Q, c.f1) + cscale(Q * Q, c.f2);
}

// field-multi.h:90-178 DexpiQ
inline M3 dexpiQ(const M3& Q, const M3& DQ) {
    CH c = ch_coeffs(Q, true);
    if (c.trivial) return zero3();
    const M3 one = unit3();
    const M3 QQ = Q * Q;
    const M3 B1 = cscale(one, c.b10) + cscale(Q, c.b11) + cscale(QQ, c.b12);
    const M3 B2 = cscale(one, c.b20) + cscale(Q, c.b21) + cscale(QQ, c.b22);
    return cscale(B1, tr(Q * DQ)) + cscale(B2, tr(QQ * DQ)) + cscale(DQ, c.f1) + cscale(DQ * Q, c.f2) +
           cscale(Q * DQ, c.f2);
}

// field-multi.h:180-269 compute_Lambda
inline M3 compute_lambda(const M3& Q, const M3& SigmaP, const M3& U) {
    CH c = ch_coeffs(Q, true);
    if (c.trivial) return zero3();
    const M3 one = unit3();
    const M3 QQ = Q * Q;
    const M3 B1 = cscale(one, c.b10) + cscale(Q, c.b11) + cscale(QQ, c.b12);
    const M3 B2 = cscale(one, c.b20) + cscale(Q, c.b21) + cscale(QQ, c.b22);
    const M3 USP = U * SigmaP;
    const M3 Gamma = cscale(Q, tr(SigmaP * B1 * U)) + cscale(QQ, tr(SigmaP * B2 * U)) + cscale(USP, c.f1) +
                     cscale(Q * USP, c.f2) + cscale(USP * Q, c.f2);
    return hermitian_traceless(Gamma);
}

// ---------------------------------------------------------------- lattice
struct Lat {
    int L[4];
    long V;
    explicit Lat(const int d[4]) {
        V = 1;
        for (int i = 0; i < 4; i++) { L[i] = d[i]; V *= d[i]; }
    }
    long idx(const int x[4]) const {
        return x[0] + (long)L[0] * (x[1] + (long)L[1] * (x[2] + (long)L[2] * x[3]));
    }
    void coord(long s, int x[4]) const {
        for (int i = 0; i < 4; i++) { x[i] = (int)(s % L[i]); s /= L[i]; }
    }
    void regularize(int x[4]) const {
        for (int i = 0; i < 4; i++) x[i] = ((x[i] % L[i]) + L[i]) % L[i];
    }
};

struct Field {
    const Lat* lat;
    double* p;
    M3& at(long s, int mu) const { return *reinterpret_cast<M3*>(p + 18 * (4 * s + mu)); }
    M3& at(const int x[4], int mu) const {
        int y[4] = {x[0], x[1], x[2], x[3]};
        lat->regularize(y);
        return at(lat->idx(y), mu);
    }
};

// double-double values: global sums keep (hi, lo) until Delta H is formed
struct DD {
    double hi, lo;
};
inline DD two_sum(double a, double b) {
    const double s = a + b;
    const double bp = s - a;
    return DD{s, (a - (s - bp)) + (b - bp)};
}
inline DD dd_add(DD a, DD b) {
    DD s = two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return two_sum(s.hi, s.lo);
}
inline DD dd_neg(DD a) { return DD{-a.hi, -a.lo}; }
inline DD dd_mul(DD a, double b) {
    const double p = a.hi * b;
    const double e = std::fma(a.hi, b, -p);
    return two_sum(p, e + a.lo * b);
}
inline double dd_val(DD a) { return a.hi + a.lo; }

// double-double accumulation over a per-site array, in site order
DD dd_sum(const std::vector<double>& a) {
    DD acc{0.0, 0.0};
    for (double x : a) {
        DD s = two_sum(acc.hi, x);
        s.lo += acc.lo;
        acc = two_sum(s.hi, s.lo);
    }
    return acc;
}

// field-matrix.h:102-131 get_path_ordered_product (USE_SINGLE_NODE periodic wrap)
M3 path_product(const Field& f, const int x[4], const int* dir, int n) {
    M3 m = unit3();
    int y[4] = {x[0], x[1], x[2], x[3]};
    for (int i = 0; i < n; i++) {
        const int d = dir[i];
        if (d < 4) {
            f.lat->regularize(y);
            m = m * f.at(f.lat->idx(y), d);
            y[d]++;
        } else {
            y[d - 4]--;
            f.lat->regularize(y);
            m = m * dag(f.at(f.lat->idx(y), d - 4));
        }
    }
    return m;
}

// field-hmc.h:203-242 get_staple_dagger
M3 staple_dagger(const Field& f, const int x[4], int mu) {
    M3 s = zero3();
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        int d1[3] = {nu, mu, nu + 4};
        s += path_product(f, x, d1, 3);
        int d2[3] = {nu + 4, mu, nu};
        s += path_product(f, x, d2, 3);
    }
    return dag(s);
}

// field-hmc.h:137-201 get_rectangular_dagger
M3 rect_dagger(const Field& f, const int x[4], int mu) {
    M3 s = zero3();
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        const int paths[6][5] = {{nu, mu, mu, nu + 4, mu + 4},     {nu + 4, mu, mu, nu, mu + 4},
                                 {nu, nu, mu, nu + 4, nu + 4},     {nu + 4, nu + 4, mu, nu, nu},
                                 {mu + 4, nu, mu, mu, nu + 4},     {mu + 4, nu + 4, mu, mu, nu}};
        for (int p = 0; p < 6; p++) s += path_product(f, x, paths[p], 5);
    }
    return dag(s);
}

// field-hmc.h:262-269 get_extended_staple_dagger (Wilson: plaquette staple only)
M3 action_staple_dagger(const Field& f, const int x[4], int mu, const mo_params* p) {
    if (p->action == 1) {
        const double c0 = 1 - 8. * p->c1;
        return staple_dagger(f, x, mu) * c0 + rect_dagger(f, x, mu) * p->c1;
    }
    return staple_dagger(f, x, mu);
}

// field-hmc.h:309-337 is_constrained
int is_constrained(const int x[4], int mu, int mag) {
    if (!mag) return 0;
    bool c = true;
    for (int i = 0; i < 4; i++) {
        if (i == mu) continue;
        c = c && (x[i] % mag == 0);
    }
    if (c) {
        if (x[mu] % mag == mag - 1) return 100;
        if (x[mu] % mag == 0) return 10;
        return 1;
    }
    return 0;
}

// field-matrix.h:202-221 get_plaq
double site_plaq(const Field& f, const int x[4]) {
    double ret = 0.0;
    for (int mu = 0; mu < 4; mu++)
        for (int nu = 0; nu < mu; nu++) {
            int xm[4] = {x[0], x[1], x[2], x[3]}; xm[mu]++;
            int xn[4] = {x[0], x[1], x[2], x[3]}; xn[nu]++;
            const M3 m = f.at(x, mu) * f.at(xm, nu);
            const M3 n = dag(f.at(x, nu) * f.at(xn, mu));
            ret += retr(m * n);
        }
    return ret;
}

// field-matrix.h:249-297 get_rectangular
double site_rect(const Field& f, const int x[4]) {
    double sum = 0.0;
    for (int mu = 0; mu < 4; mu++)
        for (int nu = 0; nu < mu; nu++) {
            int x1m[4] = {x[0], x[1], x[2], x[3]}; x1m[mu]++;
            int x1n[4] = {x[0], x[1], x[2], x[3]}; x1n[nu]++;
            int x2m[4] = {x[0], x[1], x[2], x[3]}; x2m[mu] += 2;
            int x2n[4] = {x[0], x[1], x[2], x[3]}; x2n[nu] += 2;
            int x11[4] = {x[0], x[1], x[2], x[3]}; x11[mu]++; x11[nu]++;
            M3 m = dag(f.at(x, mu) * f.at(x1m, nu) * f.at(x11, nu));
            sum += retr(f.at(x, nu) * f.at(x1n, nu) * f.at(x2n, mu) * m);
            m = dag(f.at(x, mu) * f.at(x1m, mu) * f.at(x2m, nu));
            sum += retr(f.at(x, nu) * f.at(x1n, mu) * f.at(x11, mu) * m);
        }
    return sum;
}

void plaq_rect_sums(const Field& f, DD out[2], bool with_rect) {
    const Lat& lat = *f.lat;
    std::vector<double> ps(lat.V), rs(with_rect ? lat.V : 0);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        ps[s] = site_plaq(f, x);
        if (with_rect) rs[s] = site_rect(f, x);
    }
    out[0] = dd_sum(ps);
    out[1] = with_rect ? dd_sum(rs) : DD{0.0, 0.0};
}

// ---------------------------------------------------------------- stout
// Thin-link isotropic stout level (hep-lat/0311018 eq. 1-3 with the reference's
// get_Q convention, field-multi.h:32-39): Q = TA(stp U^dag) * (-i rho),
// U' = expiQ(Q) U, stp = sum of the six plaquette staples of the link.
struct StoutLevels {
    std::vector<std::vector<double>> U;  // U[0] = thin ... U[n] = fully smeared
    std::vector<std::vector<double>> Q;  // Q[k]: stout exponent of level k -> k+1
};

void stout_level(const Lat& lat, const double* Uin, double* Uout, double* Qout, double rho) {
    Field fi{&lat, const_cast<double*>(Uin)};
    Field fo{&lat, Uout};
    Field fq{&lat, Qout};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        for (int mu = 0; mu < 4; mu++) {
            const M3 stp = dag(staple_dagger(fi, x, mu));
            M3 Om = ta(stp * dag(fi.at(s, mu)));
            const M3 Q = cscale(Om, cplx(0.0, -rho));
            fq.at(s, mu) = Q;
            fo.at(s, mu) = expiQ(Q) * fi.at(s, mu);
        }
    }
}

StoutLevels stout_all(const Lat& lat, const double* U0, const mo_params* p) {
    StoutLevels st;
    const size_t n = (size_t)lat.V * 72;
    st.U.emplace_back(U0, U0 + n);
    for (int k = 0; k < p->n_stout; k++) {
        st.U.emplace_back(n);
        st.Q.emplace_back(n);
        stout_level(lat, st.U[k].data(), st.U[k + 1].data(), st.Q[k].data(), p->rho);
    }
    return st;
}

// One loop term of d/dU of ReTr(stp(y,nu_o) U^dag(y,nu_o) Lambda(y,nu_o)), for the
// target link at position `pos` (0..2) of the staple of owner (y, nu_o) that
// goes through direction `side` with `sign` (+1: upper, -1: lower staple).
// Returns the contribution to Z(target) as derived from Re Tr(dU Z).
M3 insertion_term(const Field& fu, const Field& fl, const int y[4], int nu_o, int side, int sign, int pos,
                  double rho) {
    M3 seq[5];
    int a[4] = {y[0], y[1], y[2], y[3]};
    bool dagged[3];
    if (sign > 0) {
        int b[4] = {a[0], a[1], a[2], a[3]}; b[side]++;
        int c[4] = {a[0], a[1], a[2], a[3]}; c[nu_o]++;
        seq[0] = fu.at(a, side); dagged[0] = false;
        seq[1] = fu.at(b, nu_o); dagged[1] = false;
        seq[2] = dag(fu.at(c, side)); dagged[2] = true;
    } else {
        int b[4] = {a[0], a[1], a[2], a[3]}; b[side]--;
        int c[4] = {b[0], b[1], b[2], b[3]}; c[nu_o]++;
        seq[0] = dag(fu.at(b, side)); dagged[0] = true;
        seq[1] = fu.at(b, nu_o); dagged[1] = false;
        seq[2] = fu.at(c, side); dagged[2] = false;
    }
    seq[3] = dag(fu.at(a, nu_o));
    seq[4] = fl.at(a, nu_o);
    M3 R = unit3();
    for (int k = pos + 1; k < 5; k++) R = R * seq[k];
    for (int k = 0; k < pos; k++) R = R * seq[k];
    if (dagged[pos]) return cscale(dag(R), cplx(0.0, rho));
    return cscale(R, cplx(0.0, -rho));
}

// Chain rule of one stout level: Z holds dS/dU' on entry (Re Tr(dU' Z) form),
// dS/dU on exit.  Terms: Z' e^{iQ}, i C^dag Lambda, and the six staple insertions
// per direction (hep-lat/0311018 eq. 75 with the reference's Lambda,
// field-multi.h:267-268).
void stout_backward(const Lat& lat, const double* Uk, const double* Qk, double* Z, double rho) {
    const size_t n = (size_t)lat.V * 72;
    std::vector<double> lam(n), znew(n);
    Field fu{&lat, const_cast<double*>(Uk)};
    Field fq{&lat, const_cast<double*>(Qk)};
    Field fz{&lat, Z};
    Field fl{&lat, lam.data()};
    Field fn{&lat, znew.data()};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++)
        for (int mu = 0; mu < 4; mu++) fl.at(s, mu) = compute_lambda(fq.at(s, mu), fz.at(s, mu), fu.at(s, mu));
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        for (int mu = 0; mu < 4; mu++) {
            const M3 stp = dag(staple_dagger(fu, x, mu));
            M3 acc = fz.at(s, mu) * expiQ(fq.at(s, mu));
            acc += cscale(dag(stp) * fl.at(s, mu), cplx(0.0, rho));
            for (int nu = 0; nu < 4; nu++) {
                if (nu == mu) continue;
                int y[4];
                // (1) owner (x-nu, mu), upper staple through nu: target is its middle link
                std::copy(x, x + 4, y); y[nu]--;
                acc += insertion_term(fu, fl, y, mu, nu, +1, 1, rho);
                // (2) owner (x+nu, mu), lower staple through nu: middle link
                std::copy(x, x + 4, y); y[nu]++;
                acc += insertion_term(fu, fl, y, mu, nu, -1, 1, rho);
                // (3) owner (x, nu), upper staple through mu: first link
                std::copy(x, x + 4, y);
                acc += insertion_term(fu, fl, y, nu, mu, +1, 0, rho);
                // (4) owner (x-nu, nu), upper staple through mu: third link (daggered)
                std::copy(x, x + 4, y); y[nu]--;
                acc += insertion_term(fu, fl, y, nu, mu, +1, 2, rho);
                // (5) owner (x+mu, nu), lower staple through mu: first link (daggered)
                std::copy(x, x + 4, y); y[mu]++;
                acc += insertion_term(fu, fl, y, nu, mu, -1, 0, rho);
                // (6) owner (x+mu-nu, nu), lower staple through mu: third link
                std::copy(x, x + 4, y); y[mu]++; y[nu]--;
                acc += insertion_term(fu, fl, y, nu, mu, -1, 2, rho);
            }
            fn.at(s, mu) = acc;
        }
    }
    std::memcpy(Z, znew.data(), n * sizeof(double));
}

// ---------------------------------------------------------------- force
// Left-derivative matrix M(x,mu) = U(x,mu) Z(x,mu) of the (smeared) action for
// every link, with dS = -beta/3 Re Tr(dU Z).  Thin links: Z = extended staple
// dagger (field-hmc.h:395-396).
void derivative_fields(const mo_params* p, const Lat& lat, const double* U, std::vector<double>& Zthin) {
    const size_t n = (size_t)lat.V * 72;
    StoutLevels st = stout_all(lat, U, p);
    Zthin.assign(n, 0.0);
    Field ftop{&lat, st.U.back().data()};
    Field fz{&lat, Zthin.data()};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        for (int mu = 0; mu < 4; mu++) fz.at(s, mu) = action_staple_dagger(ftop, x, mu, p);
    }
    for (int k = p->n_stout - 1; k >= 0; k--) stout_backward(lat, st.U[k].data(), st.Q[k].data(), Zthin.data(), p->rho);
}

// field-hmc.h:339-425 get_force, generalised to a smeared action through Z.
void force(const mo_params* p, const double* U, double* F) {
    Lat lat(p->dims);
    Field fu{&lat, const_cast<double*>(U)};
    Field ff{&lat, F};
    const cplx ib3(0.0, p->beta / 3.0);
    if (p->n_stout == 0) {
        // literal restatement of the thin-link branch
#pragma omp parallel for schedule(static)
        for (long s = 0; s < lat.V; s++) {
            int x[4];
            lat.coord(s, x);
            for (int mu = 0; mu < 4; mu++) {
                M3 t;
                switch (is_constrained(x, mu, p->mag)) {
                    case 0: t = fu.at(s, mu) * action_staple_dagger(fu, x, mu, p); break;
                    case 1:
                    case 10: {
                        int y[4] = {x[0], x[1], x[2], x[3]}; y[mu]++;
                        const M3 s1 = action_staple_dagger(fu, x, mu, p);
                        const M3 s2 = action_staple_dagger(fu, y, mu, p);
                        t = fu.at(y, mu) * s2 - s1 * fu.at(s, mu);
                        break;
                    }
                    default: t = zero3(); break;
                }
                ff.at(s, mu) = cscale(ta(t), ib3);
            }
        }
        return;
    }
    std::vector<double> Z;
    derivative_fields(p, lat, U, Z);
    Field fz{&lat, Z.data()};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        for (int mu = 0; mu < 4; mu++) {
            M3 t;
            switch (is_constrained(x, mu, p->mag)) {
                case 0: t = fu.at(s, mu) * fz.at(s, mu); break;
                case 1:
                case 10: {
                    int y[4] = {x[0], x[1], x[2], x[3]}; y[mu]++;
                    t = fu.at(y, mu) * fz.at(y, mu) - fz.at(s, mu) * fu.at(s, mu);
                    break;
                }
                default: t = zero3(); break;
            }
            ff.at(s, mu) = cscale(ta(t), ib3);
        }
    }
}

// field-hmc.h:427-440 evolve_momentum
void evolve_momentum(const Lat& lat, double* P, const double* F, double dt, double m) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < lat.V * 72; i++) P[i] += F[i] * dt * m;
}

// field-hmc.h:442-482 evolve_gauge_field
void evolve_gauge(const mo_params* p, const Lat& lat, double* U, const double* P, double dt) {
    Field fu{&lat, U};
    Field fp{&lat, const_cast<double*>(P)};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        for (int mu = 0; mu < 4; mu++) {
            int y[4] = {x[0], x[1], x[2], x[3]}; y[mu]--;
            M3& g = fu.at(s, mu);
            switch (is_constrained(x, mu, p->mag)) {
                case 0: g = expiQ(fp.at(s, mu) * dt) * g; break;
                case 1: g = expiQ(fp.at(y, mu) * dt) * g * expiQ(fp.at(s, mu) * -dt); break;
                case 10: g = g * expiQ(fp.at(s, mu) * -dt); break;
                case 100: g = expiQ(fp.at(y, mu) * dt) * g; break;
            }
        }
    }
}

// field-matrix.h:83-100 reunitarize
double reunitarize(const Lat& lat, double* U) {
    double maxdev = 0.0;
    for (long i = 0; i < lat.V * 4; i++) {
        M3& m = *reinterpret_cast<M3*>(U + 18 * i);
        const M3 old = m;
        bool all_zero = true;
        for (int k = 0; k < 12; k++) all_zero = all_zero && (0.0 == m.v[k]);
        if (!all_zero) unitarize(m);
        maxdev = std::max(maxdev, fnorm(m - old));
    }
    return maxdev;
}

// field-hmc.h:589-644 get_hamiltonian (kinetic part, case 100 excluded)
DD kinetic(const mo_params* p, const Lat& lat, const double* P) {
    Field fp{&lat, const_cast<double*>(P)};
    std::vector<double> ks(lat.V);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        double acc = 0.0;
        for (int mu = 0; mu < 4; mu++) {
            if (is_constrained(x, mu, p->mag) == 100) continue;
            const M3& m = fp.at(s, mu);
            acc += retr(m * m);
        }
        ks[s] = acc;
    }
    return dd_mul(dd_sum(ks), 0.5);
}

// action of the (smeared) field: out = {sum ReTr plaq, sum ReTr rect, S}
// (field-hmc.h:632-639: S = beta/3 [(1 - 8 c1)(-sum plaq) + c1 (-sum rect)])
void action(const mo_params* p, const Lat& lat, const double* U, DD out[3]) {
    std::vector<double> top;
    const double* Ut = U;
    if (p->n_stout > 0) {
        StoutLevels st = stout_all(lat, U, p);
        top = st.U.back();
        Ut = top.data();
    }
    Field f{&lat, const_cast<double*>(Ut)};
    DD pr[2];
    plaq_rect_sums(f, pr, true);
    out[0] = pr[0];
    out[1] = pr[1];
    DD t;
    if (p->action == 1) t = dd_add(dd_mul(dd_neg(pr[0]), 1. - 8. * p->c1), dd_mul(dd_neg(pr[1]), p->c1));
    else t = dd_neg(pr[0]);
    out[2] = dd_mul(t, p->beta / 3.);
}

// field-hmc.h:525-567 force_gradient_integrator; field-hmc.h:569-587 leap_frog_integrator
void integrate(const mo_params* p, const Lat& lat, double* U, double* P, double* maxdev) {
    const size_t n = (size_t)lat.V * 72;
    std::vector<double> F(n), Uaux(n);
    const double dt = p->tau / p->n_steps;
    if (p->integrator == 1) {
        evolve_gauge(p, lat, U, P, dt / 2.);
        for (int i = 0; i < p->n_steps; i++) {
            force(p, U, F.data());
            evolve_momentum(lat, P, F.data(), dt, 1.0);
            if (i < p->n_steps - 1) evolve_gauge(p, lat, U, P, dt);
            else evolve_gauge(p, lat, U, P, dt / 2.);
        }
        if (maxdev) *maxdev = 0.0;
        return;
    }
    const double alpha = (3. - std::sqrt(3.)) * dt / 6.;
    const double beta = dt / std::sqrt(3.);
    const double gamma = (2. - std::sqrt(3.)) * dt * dt / 12.;
    evolve_gauge(p, lat, U, P, alpha);
    for (int i = 0; i < p->n_steps; i++) {
        for (int half = 0; half < 2; half++) {
            force(p, U, F.data());
            std::memcpy(Uaux.data(), U, n * sizeof(double));
            evolve_gauge(p, lat, Uaux.data(), F.data(), gamma);
            force(p, Uaux.data(), F.data());
            evolve_momentum(lat, P, F.data(), 0.5 * dt, 1.0);
            if (half == 0) evolve_gauge(p, lat, U, P, beta);
        }
        if (i < p->n_steps - 1) evolve_gauge(p, lat, U, P, 2. * alpha);
        else evolve_gauge(p, lat, U, P, alpha);
    }
    const double d = reunitarize(lat, U);
    if (maxdev) *maxdev = d;
}

// ---------------------------------------------------------------- RNG
inline void philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

enum { PURPOSE_MOMENTA = 1, PURPOSE_HOT = 2, PURPOSE_ACCEPT = 3 };

inline void gauss4(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, double g[4]) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const uint32_t ctr[4] = {c0, c1, c2, c3};
    uint32_t o[4];
    philox(ctr, key, o);
    for (int k = 0; k < 2; k++) {
        const double u1 = ((double)o[2 * k] + 0.5) * 2.3283064365386963e-10;
        const double u2 = ((double)o[2 * k + 1] + 0.5) * 2.3283064365386963e-10;
        const double r = std::sqrt(-2.0 * std::log(u1));
        g[2 * k] = r * std::cos(6.283185307179586 * u2);
        g[2 * k + 1] = r * std::sin(6.283185307179586 * u2);
    }
}

// su(3) generators T_a = lambda_a / sqrt(2) (field-hmc.h:30-69)
std::vector<M3> generators() {
    std::vector<M3> T(8, zero3());
    const double s2 = 1. / std::sqrt(2.);
    set(T[0], 0, 1, 1.0); set(T[0], 1, 0, 1.0);
    set(T[1], 0, 1, cplx(0, -1)); set(T[1], 1, 0, cplx(0, 1));
    set(T[2], 0, 0, 1.0); set(T[2], 1, 1, -1.0);
    set(T[3], 0, 2, 1.0); set(T[3], 2, 0, 1.0);
    set(T[4], 0, 2, cplx(0, -1)); set(T[4], 2, 0, cplx(0, 1));
    set(T[5], 1, 2, 1.0); set(T[5], 2, 1, 1.0);
    set(T[6], 1, 2, cplx(0, -1)); set(T[6], 2, 1, cplx(0, 1));
    set(T[7], 0, 0, 1.0); set(T[7], 1, 1, 1.0); set(T[7], 2, 2, -2.0);
    for (int a = 0; a < 7; a++) T[a] = T[a] * s2;
    T[7] = T[7] * (1. / std::sqrt(6.));
    return T;
}

}  // namespace

// ====================================================================== C API
extern "C" {

void mo_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int mo_get_threads(void) { return omp_get_max_threads(); }

void mo_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

// Haar-random SU(3) hot start: Gram-Schmidt of two complex Gaussian rows, row 2
// from their cross product.
void mo_gen_hot(const int dims[4], uint64_t seed, double* U) {
    Lat lat(dims);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < lat.V * 4; l++) {
        double g[12];
        for (int j = 0; j < 3; j++) gauss4(seed, (uint32_t)l, (uint32_t)j, 0u, PURPOSE_HOT, g + 4 * j);
        M3 m = zero3();
        for (int k = 0; k < 3; k++) {
            set(m, 0, k, cplx(g[2 * k], g[2 * k + 1]));
            set(m, 1, k, cplx(g[6 + 2 * k], g[6 + 2 * k + 1]));
        }
        unitarize(m);
        std::memcpy(U + 18 * l, m.v, sizeof(m.v));
    }
}

// field-hmc.h:675-693 init_momentum: P = sum_a T_a xi_a, xi ~ N(0,1), order mu then a
void mo_gen_momenta(const int dims[4], uint64_t seed, uint64_t traj, double* P) {
    Lat lat(dims);
    static const std::vector<M3> T = generators();
#pragma omp parallel for schedule(static)
    for (long l = 0; l < lat.V * 4; l++) {
        double xi[8];
        for (int j = 0; j < 2; j++) gauss4(seed, (uint32_t)l, (uint32_t)j, (uint32_t)traj, PURPOSE_MOMENTA, xi + 4 * j);
        M3 m = zero3();
        for (int a = 0; a < 8; a++) m += T[a] * xi[a];
        std::memcpy(P + 18 * l, m.v, sizeof(m.v));
    }
}

double mo_gen_uniform(uint64_t seed, uint64_t traj) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const uint32_t ctr[4] = {0u, 0u, (uint32_t)traj, PURPOSE_ACCEPT};
    uint32_t o[4];
    philox(ctr, key, o);
    return ((double)(o[0] >> 5) * 67108864.0 + (double)(o[1] >> 6)) * (1.0 / 9007199254740992.0);
}

void mo_expiQ(const double* Q, double* out) {
    M3 q; std::memcpy(q.v, Q, sizeof(q.v));
    const M3 r = expiQ(q);
    std::memcpy(out, r.v, sizeof(r.v));
}
void mo_dexpiQ(const double* Q, const double* DQ, double* out) {
    M3 q, d; std::memcpy(q.v, Q, sizeof(q.v)); std::memcpy(d.v, DQ, sizeof(d.v));
    const M3 r = dexpiQ(q, d);
    std::memcpy(out, r.v, sizeof(r.v));
}
void mo_compute_lambda(const double* Q, const double* SigmaP, const double* U, double* out) {
    M3 q, s, u;
    std::memcpy(q.v, Q, sizeof(q.v)); std::memcpy(s.v, SigmaP, sizeof(s.v)); std::memcpy(u.v, U, sizeof(u.v));
    const M3 r = compute_lambda(q, s, u);
    std::memcpy(out, r.v, sizeof(r.v));
}
void mo_unitarize(double* M) {
    M3 m; std::memcpy(m.v, M, sizeof(m.v));
    unitarize(m);
    std::memcpy(M, m.v, sizeof(m.v));
}
void mo_ta(const double* M, double* out) {
    M3 m; std::memcpy(m.v, M, sizeof(m.v));
    const M3 r = ta(m);
    std::memcpy(out, r.v, sizeof(r.v));
}

void mo_plaq_rect(const int dims[4], const double* U, double out[2]) {
    Lat lat(dims);
    Field f{&lat, const_cast<double*>(U)};
    DD pr[2];
    plaq_rect_sums(f, pr, true);
    out[0] = dd_val(pr[0]);
    out[1] = dd_val(pr[1]);
}

// field-matrix.h:387-389 avg_plaquette
double mo_avg_plaquette(const int dims[4], const double* U) {
    Lat lat(dims);
    Field f{&lat, const_cast<double*>(U)};
    DD pr[2];
    plaq_rect_sums(f, pr, false);
    return dd_val(pr[0]) / (18. * lat.V);
}

void mo_action(const mo_params* p, const double* U, double out[3]) {
    Lat lat(p->dims);
    DD a[3];
    action(p, lat, U, a);
    for (int k = 0; k < 3; k++) out[k] = dd_val(a[k]);
}

double mo_kinetic(const mo_params* p, const double* P) {
    Lat lat(p->dims);
    return dd_val(kinetic(p, lat, P));
}

void mo_staple_dagger(const mo_params* p, const double* U, double* V) {
    Lat lat(p->dims);
    Field fu{&lat, const_cast<double*>(U)};
    Field fv{&lat, V};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        for (int mu = 0; mu < 4; mu++) fv.at(s, mu) = action_staple_dagger(fu, x, mu, p);
    }
}

void mo_force(const mo_params* p, const double* U, double* F) { force(p, U, F); }

void mo_evolve_gauge(const mo_params* p, double* U, const double* P, double dt) {
    Lat lat(p->dims);
    evolve_gauge(p, lat, U, P, dt);
}

void mo_evolve_momentum(const int dims[4], double* P, const double* F, double dt, double m) {
    Lat lat(dims);
    evolve_momentum(lat, P, F, dt, m);
}

double mo_reunitarize(const int dims[4], double* U) {
    Lat lat(dims);
    return reunitarize(lat, U);
}

void mo_integrate(const mo_params* p, double* U, double* P, double* reunit_maxdev) {
    Lat lat(p->dims);
    integrate(p, lat, U, P, reunit_maxdev);
}

namespace {
// {kinetic, potential, plaq_sum, rect_sum} in double-double
struct HamDD {
    DD kin, pot, plaq, rect;
};
HamDD hamiltonian_dd(const mo_params* p, const Lat& lat, const double* U, const double* P) {
    DD a[3];
    action(p, lat, U, a);
    return HamDD{kinetic(p, lat, P), a[2], a[0], a[1]};
}
}  // namespace

// out = {H, kinetic, potential, plaq_sum, rect_sum}
void mo_hamiltonian(const mo_params* p, const double* U, const double* P, double out[5]) {
    Lat lat(p->dims);
    const HamDD h = hamiltonian_dd(p, lat, U, P);
    out[0] = dd_val(dd_add(h.kin, h.pot));
    out[1] = dd_val(h.kin);
    out[2] = dd_val(h.pot);
    out[3] = dd_val(h.plaq);
    out[4] = dd_val(h.rect);
}

// One trajectory of field-hmc.h:806-843 run_chmc with given momenta and uniform;
// accept = 1 selects the trajectory-level demon of field-demon.h:173-186.
void mo_trajectory(const mo_params* p, int traj_index, double* U, const double* P, double uniform,
                   double demon[2], mo_traj* res) {
    Lat lat(p->dims);
    const size_t n = (size_t)lat.V * 72;
    std::vector<double> Pw(P, P + n), Uold(U, U + n);
    const HamDD a = hamiltonian_dd(p, lat, U, Pw.data());
    double maxdev = 0.0;
    integrate(p, lat, U, Pw.data(), &maxdev);
    const HamDD b = hamiltonian_dd(p, lat, U, Pw.data());
    res->h_old = dd_val(dd_add(a.kin, a.pot)); res->kin_old = dd_val(a.kin); res->pot_old = dd_val(a.pot);
    res->plaq_old = dd_val(a.plaq); res->rect_old = dd_val(a.rect);
    res->h_new = dd_val(dd_add(b.kin, b.pot)); res->kin_new = dd_val(b.kin); res->pot_new = dd_val(b.pot);
    res->plaq_new = dd_val(b.plaq); res->rect_new = dd_val(b.rect);
    // Delta H from the compensated parts: (K1 - K0) + (S1 - S0)
    const double dh = dd_val(dd_add(dd_add(b.kin, dd_neg(a.kin)), dd_add(b.pot, dd_neg(a.pot))));
    res->delta_h = dh;
    res->uniform = uniform;
    res->reunit_maxdev = maxdev;
    bool acc;
    if (p->accept == 1) {
        // demon energies are in units of -sum ReTr (field-demon.h:152-175)
        const double ds0 = -dd_val(dd_add(b.plaq, dd_neg(a.plaq)));
        const double ds1 = -dd_val(dd_add(b.rect, dd_neg(a.rect)));
        const double e0 = demon[0] - ds0, e1 = demon[1] - ds1;
        acc = e0 > -p->e_max && e0 < p->e_max && e1 > -p->e_max && e1 < p->e_max;
        if (acc) { demon[0] = e0; demon[1] = e1; }
    } else {
        acc = uniform < std::exp(-dh);
        if (traj_index < p->n_forced) acc = true;
    }
    res->demon[0] = demon[0];
    res->demon[1] = demon[1];
    res->accept = acc ? 1 : 0;
    if (!acc) std::memcpy(U, Uold.data(), n * sizeof(double));
    res->avg_plaquette = mo_avg_plaquette(p->dims, U);
}

void mo_run(const mo_params* p, uint64_t seed, int n_traj, double* U, mo_traj* res) {
    Lat lat(p->dims);
    std::vector<double> P((size_t)lat.V * 72);
    double demon[2] = {0.0, 0.0};
    for (int i = 0; i < n_traj; i++) {
        mo_gen_momenta(p->dims, seed, (uint64_t)i, P.data());
        const double u = mo_gen_uniform(seed, (uint64_t)i);
        mo_trajectory(p, i, U, P.data(), u, demon, res + i);
    }
}

// levels: (n_stout + 1) consecutive fields, level 0 = copy of U
void mo_stout_forward(const mo_params* p, const double* U, double* levels) {
    Lat lat(p->dims);
    StoutLevels st = stout_all(lat, U, p);
    const size_t n = (size_t)lat.V * 72;
    for (size_t k = 0; k < st.U.size(); k++) std::memcpy(levels + k * n, st.U[k].data(), n * sizeof(double));
}

// field-wloop.h:26-99 wilson_loop / avg_wilson_loop
double mo_wilson_loop(const int dims[4], const double* U, const int r[3], int T) {
    Lat lat(dims);
    Field f{&lat, const_cast<double*>(U)};
    std::vector<int> rl(r, r + 3);
    std::sort(rl.begin(), rl.end());
    std::vector<std::vector<int>> perm;
    do { perm.push_back(rl); } while (std::next_permutation(rl.begin(), rl.end()));
    std::vector<double> ws(lat.V);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        double acc = 0.0;
        for (const auto& pr : perm) {
            std::vector<int> dir;
            for (int i = 0; i < 3; i++) for (int j = 0; j < pr[i]; j++) dir.push_back(i);
            for (int i = 0; i < T; i++) dir.push_back(3);
            for (int i = 2; i >= 0; i--) for (int j = 0; j < pr[i]; j++) dir.push_back(i + 4);
            for (int i = 0; i < T; i++) dir.push_back(7);
            acc += retr(path_product(f, x, dir.data(), (int)dir.size()));
        }
        ws[s] = acc;
    }
    return dd_val(dd_sum(ws)) / ((double)perm.size() * lat.V);
}

// field-matrix.h:407-443 check_constrained_plaquette
double mo_constrained_plaquette(const int dims[4], const double* U, int mag) {
    Lat lat(dims);
    Field f{&lat, const_cast<double*>(U)};
    long count = 0;
    double sum = 0.0;
    for (int x0 = 0; x0 < lat.L[0]; x0 += mag)
        for (int x1 = 0; x1 < lat.L[1]; x1 += mag)
            for (int x2 = 0; x2 < lat.L[2]; x2 += mag)
                for (int x3 = 0; x3 < lat.L[3]; x3 += mag) {
                    const int x[4] = {x0, x1, x2, x3};
                    for (int mu = 0; mu < 4; mu++)
                        for (int nu = 0; nu < mu; nu++) {
                            std::vector<int> dir;
                            for (int i = 0; i < mag; i++) dir.push_back(mu);
                            for (int i = 0; i < mag; i++) dir.push_back(nu);
                            for (int i = 0; i < mag; i++) dir.push_back(mu + 4);
                            for (int i = 0; i < mag; i++) dir.push_back(nu + 4);
                            count++;
                            sum += retr(path_product(f, x, dir.data(), (int)dir.size()));
                        }
                }
    return sum / (3. * count);
}

// U(x,mu) -> G(x) U(x,mu) G(x+mu)^dag, G: double[V][3][3][2]
void mo_gauge_transform(const int dims[4], double* U, const double* G) {
    Lat lat(dims);
    Field fu{&lat, U};
    std::vector<double> out((size_t)lat.V * 72);
    Field fo{&lat, out.data()};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        int x[4];
        lat.coord(s, x);
        M3 g; std::memcpy(g.v, G + 18 * s, sizeof(g.v));
        for (int mu = 0; mu < 4; mu++) {
            int y[4] = {x[0], x[1], x[2], x[3]}; y[mu]++;
            lat.regularize(y);
            M3 h; std::memcpy(h.v, G + 18 * lat.idx(y), sizeof(h.v));
            fo.at(s, mu) = g * fu.at(s, mu) * dag(h);
        }
    }
    std::memcpy(U, out.data(), out.size() * sizeof(double));
}

}  // extern "C"

// ------------------------------------------------- per-link demon sweep
namespace {

enum { PURPOSE_DEMON_SU2 = 4, PURPOSE_DEMON_SUBGROUP = 5 };

// field-staple.h:27-72 (init_chair_index) and :74-120 (init_twist_index): for every
// nu != mu and lambda not in {mu, nu}, four four-step base paths, each with mu
// inserted before step 1, 2 or 3 (72 five-step paths per mu); 0-3 forward,
// 4-7 backward.  The lists are rebuilt here step by step as the reference builds them.
std::vector<std::vector<int>> demon_paths(int mu, bool twist) {
    std::vector<std::vector<int>> out;
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        for (int la = 0; la < 4; la++) {
            if (la == nu || la == mu) continue;
            int base[4][4];
            if (!twist) {
                const int b[4][4] = {{nu, la, la + 4, nu + 4}, {nu, la + 4, la + 4, nu},
                                     {nu + 4, la, la, nu + 4}, {nu + 4, la + 4, la, nu}};
                std::memcpy(base, b, sizeof(b));
            } else {
                const int b[4][4] = {{nu, la, nu + 4, la + 4}, {nu, la + 4, nu + 4, la},
                                     {nu + 4, la, nu, la + 4}, {nu + 4, la + 4, nu, la}};
                std::memcpy(base, b, sizeof(b));
            }
            for (int k = 0; k < 4; k++)
                for (int i = 1; i < 4; i++) {
                    std::vector<int> d(base[k], base[k] + 4);
                    d.insert(d.begin() + i, mu);
                    out.push_back(d);
                }
        }
    }
    return out;
}

// field-staple.h:125-134 chair_staple_dagger / :140-149 twist_staple_dagger: the
// plain sum of the path products (no dagger, despite the name)
M3 demon_staple(const Field& f, const int x[4], const std::vector<std::vector<int>>& paths) {
    M3 acc = zero3();
    for (const auto& d : paths) acc = acc + path_product(f, x, d.data(), (int)d.size());
    return acc;
}

inline double u32(uint32_t v) { return ((double)v + 0.5) * 2.3283064365386963e-10; }

// field-matrix.h:36-65 random_su3_from_su2(small, rng): a0 uniform in [small, 1),
// a1..a3 uniform in [-1, 1) scaled to |a| = sqrt(1 - a0^2), embedded in the SU(2)
// subgroup rand_gen % 3; the draws come from Philox counters (link, sweep, hit).
M3 random_su3_from_su2(double small, uint64_t seed, uint32_t link, uint32_t sweep, uint32_t hit) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const uint32_t c1[4] = {link, sweep, hit, PURPOSE_DEMON_SU2};
    const uint32_t c2[4] = {link, sweep, hit, PURPOSE_DEMON_SUBGROUP};
    uint32_t o[4], q[4];
    philox(c1, key, o);
    philox(c2, key, q);
    const double a0 = small + (1.0 - small) * u32(o[0]);
    double a1 = -1.0 + 2.0 * u32(o[1]), a2 = -1.0 + 2.0 * u32(o[2]), a3 = -1.0 + 2.0 * u32(o[3]);
    const double norm = std::sqrt((1. - a0 * a0) / (a1 * a1 + a2 * a2 + a3 * a3));
    a1 *= norm; a2 *= norm; a3 *= norm;
    M3 m = unit3();
    int i = 0, j = 0;
    switch (q[0] % 3) {
        case 0: i = 1; j = 2; break;
        case 1: i = 0; j = 2; break;
        default: i = 0; j = 1; break;
    }
    set(m, i, i, cplx(a0, a3));
    set(m, i, j, cplx(a2, a1));
    set(m, j, i, cplx(-a2, a1));
    set(m, j, j, cplx(a0, -a3));
    return m;
}

}  // namespace

extern "C" {

// field-demon.h:25-126 demon_microcanonical on a copy of the links: sites in index
// order, mu = 0..3, plaquette / rectangle / chair / twist staples of the current
// field, two hits of random_su3_from_su2(0.9), accept iff every demon stays in
// (-E_max, E_max); after each sweep the demons are recorded and the field is
// reunitarized (field-demon.h:111).  E starts at 0 (field-demon.h:44).
void mo_demon_sweeps(const int dims[4], double* U, uint64_t seed, int n_sweeps, double e_max, double* E_trace,
                     int64_t* accept, int64_t* reject, double* reunit) {
    Lat lat(dims);
    Field f{&lat, U};
    std::vector<std::vector<int>> chairs[4], twists[4];
    for (int mu = 0; mu < 4; mu++) {
        chairs[mu] = demon_paths(mu, false);
        twists[mu] = demon_paths(mu, true);
    }
    double E[4] = {0.0, 0.0, 0.0, 0.0};
    int64_t acc = 0, rej = 0;
    for (int i = 0; i < n_sweeps; i++) {
        for (long s = 0; s < lat.V; s++) {
            int x[4];
            lat.coord(s, x);
            for (int mu = 0; mu < 4; mu++) {
                const M3 S[4] = {staple_dagger(f, x, mu), rect_dagger(f, x, mu), demon_staple(f, x, chairs[mu]),
                                 demon_staple(f, x, twists[mu])};
                for (int n = 0; n < 2; n++) {
                    const M3 m = random_su3_from_su2(0.9, seed, (uint32_t)(4 * s + mu), (uint32_t)i, (uint32_t)n);
                    M3& v = f.at(s, mu);
                    double dS[4];
                    bool ok = true;
                    for (int k = 0; k < 4; k++) {
                        dS[k] = -retr((m * v) * S[k]) + retr(v * S[k]);
                        ok = ok && E[k] - dS[k] > -e_max && E[k] - dS[k] < e_max;
                    }
                    if (ok) {
                        v = m * v;
                        for (int k = 0; k < 4; k++) E[k] -= dS[k];
                        acc++;
                    } else {
                        rej++;
                    }
                }
            }
        }
        for (int k = 0; k < 4; k++) E_trace[4 * i + k] = E[k];
        reunit[i] = reunitarize(lat, U);
    }
    *accept = acc;
    *reject = rej;
}

}  // extern "C"

// ================================================================ two-level coupling
// A fine field U_f (the lattice) and a coarse field U_c (every extent halved)
// coupled through the stout-smeared blocked links of the fine field
// (field-multi.h:22-45, 309-656, 659-683, 685-756, 758-900):
//   H = K_f + K_c + S_f(U_f) - 1/eta^2 sum_{coarse x, mu} ReTr(U_c(x,mu)^dag e^{iQ(2x,mu)} V(2x,mu)),
//   V(y,mu) = U_f(y,mu) U_f(y+mu,mu)          (get_U),
//   Q(y,mu) = -i rho TA(stp(y,mu) V(y,mu)^dag) (get_Q, stp = get_staple_rect, field-hmc.h:244-258).
// The reference reads rho and eta_sqr from globals that are not in its tree;
// here they are arguments.  Both fields are unconstrained (mag = 0).
namespace {

M3 multi_V(const Field& f, const int x[4], int mu) {  // field-multi.h:24-27 get_U
    int y[4] = {x[0], x[1], x[2], x[3]};
    y[mu]++;
    return f.at(x, mu) * f.at(y, mu);
}

M3 staple_rect(const Field& f, const int x[4], int mu) {  // field-hmc.h:244-258 get_staple_rect
    M3 s = zero3();
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        const int d1[4] = {nu, mu, mu, nu + 4};
        s += path_product(f, x, d1, 4);
        const int d2[4] = {nu + 4, mu, mu, nu};
        s += path_product(f, x, d2, 4);
    }
    return s;
}

M3 multi_Q(const Field& f, const int x[4], int mu, double rho) {  // field-multi.h:29-35 get_Q
    const M3 Omega = ta(staple_rect(f, x, mu) * dag(multi_V(f, x, mu)));
    return cscale(Omega, cplx(0.0, -rho));
}

// field-matrix.h:177-197 get_path_ordered_product_insertion (-1 marks the insertion)
M3 path_insertion(const Field& f, const int x[4], const int dir[6], const M3& ins) {
    M3 m = unit3();
    int y[4] = {x[0], x[1], x[2], x[3]};
    for (int i = 0; i < 6; i++) {
        const int d = dir[i];
        if (d == -1) {
            m = m * ins;
        } else if (d < 4) {
            m = m * f.at(y, d);
            y[d]++;
        } else {
            y[d - 4]--;
            m = m * dag(f.at(y, d - 4));
        }
    }
    return m;
}

// field-multi.h:378-407 stout_type: {type, direction}
void stout_type(const int x[4], int mu, int out[2]) {
    int cnt[4], n = 0;
    for (int i = 0; i < 4; i++)
        if (x[i] % 2 == 1) cnt[n++] = i;
    out[0] = 0; out[1] = 0;
    if (n == 0) { out[0] = 1; }
    else if (n == 1) {
        if (cnt[0] == mu) out[0] = 3;
        else { out[0] = 2; out[1] = cnt[0]; }
    } else if (n == 2) {
        if (cnt[0] == mu) { out[0] = 4; out[1] = cnt[1]; }
        else if (cnt[1] == mu) { out[0] = 4; out[1] = cnt[0]; }
    }
}

inline void halve(const int y[4], int c[4]) {
    for (int i = 0; i < 4; i++) c[i] = y[i] / 2;  // y even (possibly negative): exact
}

// field-multi.h:309-340 get_eta_energy
DD eta_energy(const Lat& lc, const Field& ff, const Field& fc, double rho, double eta_sqr) {
    std::vector<double> e(lc.V);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lc.V; s++) {
        int x[4];
        lc.coord(s, x);
        const int y[4] = {2 * x[0], 2 * x[1], 2 * x[2], 2 * x[3]};
        double acc = 0.0;
        for (int mu = 0; mu < 4; mu++) {
            const M3 Gb = expiQ(multi_Q(ff, y, mu, rho)) * multi_V(ff, y, mu);
            acc += retr(dag(fc.at(s, mu)) * Gb) / eta_sqr;
        }
        e[s] = acc;
    }
    return dd_neg(dd_sum(e));
}

// field-multi.h:659-683 get_Cforce
void coarse_force(const Lat& lc, const Field& ff, const Field& fc, double* Fc, double rho, double eta_sqr) {
    Field fo{&lc, Fc};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lc.V; s++) {
        int x[4];
        lc.coord(s, x);
        const int y[4] = {2 * x[0], 2 * x[1], 2 * x[2], 2 * x[3]};
        for (int mu = 0; mu < 4; mu++) {
            const M3 G = expiQ(multi_Q(ff, y, mu, rho)) * multi_V(ff, y, mu);
            fo.at(s, mu) = cscale(ta(fc.at(s, mu) * dag(G)), cplx(0.0, 1.0 / eta_sqr));
        }
    }
}

// field-multi.h:409-656 get_Fforce: the thin gauge force of the fine field plus the
// derivative of the coupling through V and through the blocked staples, the
// insertion paths of the reference listed per stout_type
void fine_force(const mo_params* p, const Lat& lf, const Lat& lc, const Field& ff, const Field& fc, double* Ff,
                double rho, double eta_sqr) {
    Field fo{&lf, Ff};
    const cplx ib3(0.0, p->beta / 3.0);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lf.V; s++) {
        int x[4];
        lf.coord(s, x);
        for (int mu = 0; mu < 4; mu++) {
            const M3 st = p->action == 1 ? action_staple_dagger(ff, x, mu, p) : staple_dagger(ff, x, mu);
            fo.at(s, mu) = cscale(ta(ff.at(s, mu) * st), ib3);
        }
    }
    // Lambda of every coarse link (field-multi.h:459-469)
    std::vector<double> Cl(lc.V * 72);
    Field fl{&lc, Cl.data()};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lc.V; s++) {
        int x[4];
        lc.coord(s, x);
        const int y[4] = {2 * x[0], 2 * x[1], 2 * x[2], 2 * x[3]};
        for (int mu = 0; mu < 4; mu++)
            fl.at(s, mu) = compute_lambda(multi_Q(ff, y, mu, rho), dag(fc.at(s, mu)), multi_V(ff, y, mu));
    }
    const cplx ir(0.0, rho);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lf.V; s++) {
        int x[4];
        lf.coord(s, x);
        for (int mu = 0; mu < 4; mu++) {
            M3 t = zero3();
            int sx[4] = {x[0], x[1], x[2], x[3]};
            sx[mu]++;  // every insertion path starts at x + mu
            int tn[2];
            stout_type(x, mu, tn);
            int y[4], c[4];
            auto set_y = [&](int d1, int k1, int d2, int k2) {
                for (int i = 0; i < 4; i++) y[i] = x[i];
                if (d1 >= 0) y[d1] += k1;
                if (d2 >= 0) y[d2] += k2;
                halve(y, c);
            };
            switch (tn[0]) {
                case 1: {
                    int z[4] = {x[0], x[1], x[2], x[3]};
                    z[mu]++;
                    set_y(-1, 0, -1, 0);
                    t += ff.at(z, mu) * dag(fc.at(c, mu)) * expiQ(multi_Q(ff, x, mu, rho));
                    for (int nu = 0; nu < 4; nu++) {
                        if (nu == mu) continue;
                        set_y(-1, 0, -1, 0);
                        { const int d[6] = {mu, nu, mu + 4, mu + 4, nu + 4, -1};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), ir); }
                        { const int d[6] = {mu, nu + 4, mu + 4, mu + 4, nu, -1};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), ir); }
                        { const int d[6] = {nu, nu, mu + 4, nu + 4, nu + 4, -1};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, nu)), -ir); }
                        set_y(nu, -2, -1, 0);
                        { const int d[6] = {nu + 4, nu + 4, mu + 4, -1, nu, nu};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, nu)), ir); }
                    }
                    break;
                }
                case 2: {
                    const int o = tn[1];
                    set_y(o, -1, -1, 0);
                    { const int d[6] = {mu, o + 4, mu + 4, mu + 4, -1, o};
                      t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), -ir); }
                    set_y(o, 1, -1, 0);
                    { const int d[6] = {mu, o, mu + 4, mu + 4, -1, o + 4};
                      t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), -ir); }
                    break;
                }
                case 3: {
                    set_y(mu, -1, -1, 0);
                    t += dag(fc.at(c, mu)) * expiQ(multi_Q(ff, y, mu, rho)) * ff.at(y, mu);
                    for (int nu = 0; nu < 4; nu++) {
                        if (nu == mu) continue;
                        set_y(mu, -1, -1, 0);
                        { const int d[6] = {nu, mu + 4, mu + 4, nu + 4, -1, mu};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), ir); }
                        { const int d[6] = {nu + 4, mu + 4, mu + 4, nu, -1, mu};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), ir); }
                        set_y(mu, 1, -1, 0);
                        { const int d[6] = {-1, nu, nu, mu + 4, nu + 4, nu + 4};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, nu)), ir); }
                        set_y(mu, 1, nu, -2);
                        { const int d[6] = {nu + 4, nu + 4, -1, mu + 4, nu, nu};
                          t += cscale(path_insertion(ff, sx, d, fl.at(c, nu)), -ir); }
                    }
                    break;
                }
                case 4: {
                    const int o = tn[1];
                    set_y(o, -1, mu, -1);
                    { const int d[6] = {o + 4, mu + 4, mu + 4, -1, o, mu};
                      t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), -ir); }
                    set_y(o, 1, mu, -1);
                    { const int d[6] = {o, mu + 4, mu + 4, -1, o + 4, mu};
                      t += cscale(path_insertion(ff, sx, d, fl.at(c, mu)), -ir); }
                    break;
                }
                default: break;
            }
            fo.at(s, mu) += cscale(ta(ff.at(s, mu) * t), cplx(0.0, 1.0 / eta_sqr));
        }
    }
}

// K = sum ReTr(P^2) / 2 over every link (field-multi.h:270-296 get_kinetic_energy, m = 1)
DD kinetic_all(const Lat& lat, const double* P) {
    std::vector<double> ks(lat.V);
    const Field fp{&lat, const_cast<double*>(P)};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < lat.V; s++) {
        double acc = 0.0;
        for (int mu = 0; mu < 4; mu++) acc += retr(fp.at(s, mu) * fp.at(s, mu));
        ks[s] = acc;
    }
    return dd_mul(dd_sum(ks), 0.5);
}

struct MultiH {
    DD kin, fine, eta;
};
// field-multi.h:342-376 get_hamiltonian_multi
MultiH multi_hamiltonian(const mo_params* p, const Lat& lf, const Lat& lc, const double* Uf, const double* Pf,
                         const double* Uc, const double* Pc, double rho, double eta_sqr) {
    mo_params thin = *p;
    thin.n_stout = 0;
    DD a[3];
    action(&thin, lf, Uf, a);
    const Field ff{&lf, const_cast<double*>(Uf)}, fc{&lc, const_cast<double*>(Uc)};
    return MultiH{dd_add(kinetic_all(lf, Pf), kinetic_all(lc, Pc)), a[2], eta_energy(lc, ff, fc, rho, eta_sqr)};
}

// field-multi.h:685-756 force_gradient_integrator_multi
void multi_integrate(const mo_params* p, const Lat& lf, const Lat& lc, double* Uf, double* Pf, double* Uc, double* Pc,
                     double rho, double eta_sqr, double maxdev[2]) {
    mo_params q = *p;
    q.mag = 0;
    const size_t nf = (size_t)lf.V * 72, nc = (size_t)lc.V * 72;
    std::vector<double> Ff(nf), Fc(nc), Ufa(nf), Uca(nc);
    const double dt = p->tau / p->n_steps;
    const double alpha = (3. - std::sqrt(3.)) * dt / 6.;
    const double beta = dt / std::sqrt(3.);
    const double gamma = (2. - std::sqrt(3.)) * dt * dt / 12.;
    mo_params qc = q;
    for (int i = 0; i < 4; i++) qc.dims[i] = lc.L[i];
    auto forces = [&](double* uf, double* uc) {
        const Field ff{&lf, uf}, fc{&lc, uc};
        fine_force(p, lf, lc, ff, fc, Ff.data(), rho, eta_sqr);
        coarse_force(lc, ff, fc, Fc.data(), rho, eta_sqr);
    };
    auto drift = [&](double eps) {
        evolve_gauge(&q, lf, Uf, Pf, eps);
        evolve_gauge(&qc, lc, Uc, Pc, eps);
    };
    auto fg_kick = [&]() {
        forces(Uf, Uc);
        std::memcpy(Ufa.data(), Uf, nf * sizeof(double));
        std::memcpy(Uca.data(), Uc, nc * sizeof(double));
        evolve_gauge(&q, lf, Ufa.data(), Ff.data(), gamma);
        evolve_gauge(&qc, lc, Uca.data(), Fc.data(), gamma);
        forces(Ufa.data(), Uca.data());
        evolve_momentum(lf, Pf, Ff.data(), 0.5 * dt, 1.0);
        evolve_momentum(lc, Pc, Fc.data(), 0.5 * dt, 1.0);
    };
    drift(alpha);
    for (int i = 0; i < p->n_steps; i++) {
        fg_kick();
        drift(beta);
        fg_kick();
        drift(i < p->n_steps - 1 ? 2. * alpha : alpha);
    }
    maxdev[0] = reunitarize(lf, Uf);
    maxdev[1] = reunitarize(lc, Uc);
}

void coarse_dims(const int d[4], int c[4]) {
    for (int i = 0; i < 4; i++) c[i] = d[i] / 2;
}

}  // namespace

extern "C" {

// fine force Ff (fine lattice) and coarse force Fc (every extent halved)
void mo_multi_forces(const mo_params* p, double rho, double eta_sqr, const double* Uf, const double* Uc, double* Ff,
                     double* Fc) {
    int cd[4];
    coarse_dims(p->dims, cd);
    Lat lf(p->dims), lc(cd);
    const Field ff{&lf, const_cast<double*>(Uf)}, fc{&lc, const_cast<double*>(Uc)};
    fine_force(p, lf, lc, ff, fc, Ff, rho, eta_sqr);
    coarse_force(lc, ff, fc, Fc, rho, eta_sqr);
}

// out = {H, kinetic (both levels), fine gauge action, coupling energy}
void mo_multi_hamiltonian(const mo_params* p, double rho, double eta_sqr, const double* Uf, const double* Pf,
                          const double* Uc, const double* Pc, double out[4]) {
    int cd[4];
    coarse_dims(p->dims, cd);
    Lat lf(p->dims), lc(cd);
    const MultiH h = multi_hamiltonian(p, lf, lc, Uf, Pf, Uc, Pc, rho, eta_sqr);
    out[0] = dd_val(dd_add(dd_add(h.kin, h.fine), h.eta));
    out[1] = dd_val(h.kin);
    out[2] = dd_val(h.fine);
    out[3] = dd_val(h.eta);
}

// one trajectory of run_hmc_multi (field-multi.h:858-900) with given momenta and uniform;
// out = {H_old, H_new, Delta H, accept, reunit fine, reunit coarse}
void mo_multi_trajectory(const mo_params* p, double rho, double eta_sqr, int traj_index, double* Uf,
                         const double* Pf, double* Uc, const double* Pc, double uniform, double out[6]) {
    int cd[4];
    coarse_dims(p->dims, cd);
    Lat lf(p->dims), lc(cd);
    const size_t nf = (size_t)lf.V * 72, nc = (size_t)lc.V * 72;
    std::vector<double> pf(Pf, Pf + nf), pc(Pc, Pc + nc), uf0(Uf, Uf + nf), uc0(Uc, Uc + nc);
    const MultiH a = multi_hamiltonian(p, lf, lc, Uf, pf.data(), Uc, pc.data(), rho, eta_sqr);
    double dev[2];
    multi_integrate(p, lf, lc, Uf, pf.data(), Uc, pc.data(), rho, eta_sqr, dev);
    const MultiH b = multi_hamiltonian(p, lf, lc, Uf, pf.data(), Uc, pc.data(), rho, eta_sqr);
    const double dh = dd_val(dd_add(dd_add(dd_add(b.kin, dd_neg(a.kin)), dd_add(b.fine, dd_neg(a.fine))),
                                    dd_add(b.eta, dd_neg(a.eta))));
    bool acc = uniform < std::exp(-dh);
    if (traj_index < p->n_forced) acc = true;
    if (!acc) {
        std::memcpy(Uf, uf0.data(), nf * sizeof(double));
        std::memcpy(Uc, uc0.data(), nc * sizeof(double));
    }
    out[0] = dd_val(dd_add(dd_add(a.kin, a.fine), a.eta));
    out[1] = dd_val(dd_add(dd_add(b.kin, b.fine), b.eta));
    out[2] = dh;
    out[3] = acc ? 1.0 : 0.0;
    out[4] = dev[0];
    out[5] = dev[1];
}

}  // extern "C"
