// su3.cuh -- SU(3) algebra for the constrained HMC kernels (float or double).
//
// A link is a 3x3 complex matrix (cps::Matrix in the reference, field-matrix.h).
// Hermitian traceless matrices (momenta P, forces F, stout exponents Q, stout
// Lambda) travel in a compact 8-real form
//     h = (H00, H11, Re H01, Im H01, Re H02, Im H02, Re H12, Im H12),
// with H22 = -H00 - H11 and the lower triangle conjugate-symmetric.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define MAG_HD __host__ __device__ __forceinline__
#else
#define MAG_HD inline
#endif

namespace magb {

// Aligned to its size, so that one element is one 64-bit (float) or 128-bit
// (double) memory access instead of two.
template <typename T>
struct alignas(2 * sizeof(T)) cplx {
    T re, im;
};

template <typename T>
MAG_HD cplx<T> mk(T r, T i) { cplx<T> c; c.re = r; c.im = i; return c; }
template <typename T>
MAG_HD cplx<T> operator+(cplx<T> a, cplx<T> b) { return mk(a.re + b.re, a.im + b.im); }
template <typename T>
MAG_HD cplx<T> operator-(cplx<T> a, cplx<T> b) { return mk(a.re - b.re, a.im - b.im); }
template <typename T>
MAG_HD cplx<T> operator*(cplx<T> a, cplx<T> b) { return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
template <typename T>
MAG_HD cplx<T> operator*(cplx<T> a, T s) { return mk(a.re * s, a.im * s); }
template <typename T>
MAG_HD cplx<T> conj(cplx<T> a) { return mk(a.re, -a.im); }

template <typename T>
struct mat3 {
    cplx<T> e[3][3];
};

template <typename T>
struct herm8 {
    T h[8];
};

template <typename T>
MAG_HD void set_zero(mat3<T>& m) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) m.e[i][j] = mk<T>(0, 0);
}
template <typename T>
MAG_HD mat3<T> zero_mat() { mat3<T> m; set_zero(m); return m; }
template <typename T>
MAG_HD mat3<T> unit_mat() {
    mat3<T> m;
    set_zero(m);
    m.e[0][0].re = m.e[1][1].re = m.e[2][2].re = T(1);
    return m;
}

// ------------------------------------------------------------ products
// Every product is a chain of fused multiply-adds into one accumulator per
// real component: c.re <- fma(a.re, b.re, c.re), c.re <- fma(-a.im, b.im, c.re),
// ...  Written as `c += a.re*b.re - a.im*b.im` the compiler has to form the
// difference first (a multiply, an fma and an add per real component); the
// chain below is two fmas per component and term.
MAG_HD float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
MAG_HD double fmaT(double a, double b, double c) { return fma(a, b, c); }

// s (+/-)= op(a) op(b), op = conjugation when CA / CB; SUB subtracts
template <bool CA, bool CB, bool SUB, typename T>
MAG_HD void cmac(cplx<T>& s, cplx<T> a, cplx<T> b) {
    const T ar = SUB ? -a.re : a.re;
    const T ai = (SUB != CA) ? -a.im : a.im;  // sign of a.im in op(a), times the sign of the update
    const T bi = CB ? -b.im : b.im;
    s.re = fmaT(ar, b.re, s.re);
    s.re = fmaT(-ai, bi, s.re);
    s.im = fmaT(ar, bi, s.im);
    s.im = fmaT(ai, b.re, s.im);
}
// s = op(a) op(b)
template <bool CA, bool CB, typename T>
MAG_HD cplx<T> cmul(cplx<T> a, cplx<T> b) {
    const T ai = CA ? -a.im : a.im;
    const T bi = CB ? -b.im : b.im;
    cplx<T> s;
    s.re = a.re * b.re;
    s.re = fmaT(-ai, bi, s.re);
    s.im = a.re * bi;
    s.im = fmaT(ai, b.re, s.im);
    return s;
}

// ------------------------------------------------- packed FP32 (sm_100a)
// fma.rn.f32x2 does two FP32 FMAs in one instruction at the FMA pipe's rate
// for two scalar FMAs, so it saves issue slots, not pipe time.
// Complex sums s = sum_k x_k y_k are written on (re, im) pairs as
//   T = sum_k (x.re, x.re) * (y.re, y.im),   U = sum_k (x.im, x.im) * (y.im, y.re),
//   s = (T.re - U.re, T.im + U.im)   [one more packed FMA with the pair (-1, 1)]:
// one factor is broadcast (its conjugation is a sign on the broadcast value),
// the other is read as a pair in natural and swapped order; a conjugated
// paired factor flips the sign of T.im and U.re at the combine.  A term costs
// two packed FMAs instead of four scalar ones (two accumulators per element;
// the single-accumulator form s += (x.re, x.re) (y.re, y.im) + (x.im, x.im)
// (-y.im, y.re) measured slower in these kernels).  The combine is FMA-pipe
// work the scalar form does not do, so the short sums (the third-row
// reconstruction of special-unitary products, the products with a Hermitian
// factor) stay scalar: packed they measured slower.  The sums are grouped
// differently from the scalar chains, so results differ by FP32 rounding.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
#define MAG_F32X2 1
namespace f2 {
__device__ __forceinline__ float2 nat(cplx<float> a) { return make_float2(a.re, a.im); }
__device__ __forceinline__ float2 swp(cplx<float> a) { return make_float2(a.im, a.re); }
__device__ __forceinline__ float2 bc(float x) { return make_float2(x, x); }
__device__ __forceinline__ cplx<float> un(float2 v) { cplx<float> c; c.re = v.x; c.im = v.y; return c; }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// T/U accumulation of one output element: s = sum_k op(x_k) op(y_k) with the
// broadcast factor x (conjugated when CX) and the paired factor y (conjugated
// when CY); ACC = 0: c = s, 1: c += s, -1: c -= s.  N terms.
template <int N, bool CX, bool CY, int ACC>
__device__ __forceinline__ cplx<float> dot(const cplx<float>* x, const cplx<float>* y, cplx<float> c) {
    // result = T * tau + U * sigma, tau = (1, sy), sigma = (-sy, 1), sy = -1 when CY;
    // the sign of the update is folded into the broadcasts.
    constexpr float sg = ACC < 0 ? -1.f : 1.f;
    constexpr float sxi = CX ? -1.f : 1.f;
    float2 T, U;
    if (ACC != 0 && !CY) T = nat(c);  // tau = (1, 1): T carries c
#pragma unroll
    for (int k = 0; k < N; k++) {
        const float2 br = bc(sg * x[k].re), bi = bc(sg * sxi * x[k].im);
        if (k == 0 && !(ACC != 0 && !CY)) T = mul2(br, nat(y[k]));
        else T = fma2(br, nat(y[k]), T);
        if (k == 0) U = mul2(bi, swp(y[k]));
        else U = fma2(bi, swp(y[k]), U);
    }
    if (!CY) return un(fma2(U, make_float2(-1.f, 1.f), T));
    const float2 tau = make_float2(1.f, -1.f), sigma = make_float2(1.f, 1.f);
    if (ACC == 0) return un(fma2(U, sigma, mul2(T, tau)));
    return un(fma2(U, sigma, fma2(T, tau, nat(c))));
}

// rows [0, R) of c (=, +=, -=) op(a) op(b); the conjugated factor (if only
// one is) is the broadcast one
template <int R, int TA, int TB, int ACC>
__device__ __forceinline__ void gemm(mat3<float>& c, const mat3<float>& a, const mat3<float>& b) {
#pragma unroll
    for (int i = 0; i < R; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cplx<float> x[3], y[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                x[k] = TA ? a.e[k][i] : a.e[i][k];
                y[k] = TB ? b.e[j][k] : b.e[k][j];
            }
            if (TB && !TA) c.e[i][j] = dot<3, true, false, ACC>(y, x, c.e[i][j]);
            else c.e[i][j] = dot<3, TA != 0, TB != 0, ACC>(x, y, c.e[i][j]);
        }
}

}  // namespace f2
#endif

// rows [0, R) of  c = op(a) op(b)  (ACC = 0),  c += ...  (ACC = 1),  c -= ...  (ACC = -1);
// TA / TB = 1 take the adjoint of a / b
template <int R, int TA, int TB, int ACC, typename T>
MAG_HD void gemm(mat3<T>& c, const mat3<T>& a, const mat3<T>& b) {
#ifdef MAG_F32X2
    if constexpr (sizeof(T) == 4) {
        f2::gemm<R, TA, TB, ACC>(c, a, b);
        return;
    }
#endif
#pragma unroll
    for (int i = 0; i < R; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cplx<T> s;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const cplx<T> x = TA ? a.e[k][i] : a.e[i][k];
                const cplx<T> y = TB ? b.e[j][k] : b.e[k][j];
                if (k == 0 && ACC == 0) s = cmul<TA != 0, TB != 0>(x, y);
                else {
                    if (k == 0) s = c.e[i][j];
                    cmac<TA != 0, TB != 0, (ACC < 0)>(s, x, y);
                }
            }
            c.e[i][j] = s;
        }
}

// c = a * b
template <typename T>
MAG_HD mat3<T> mul(const mat3<T>& a, const mat3<T>& b) { mat3<T> c; gemm<3, 0, 0, 0>(c, a, b); return c; }
// c = a * b^dag
template <typename T>
MAG_HD mat3<T> mul_nd(const mat3<T>& a, const mat3<T>& b) { mat3<T> c; gemm<3, 0, 1, 0>(c, a, b); return c; }
// c = a^dag * b
template <typename T>
MAG_HD mat3<T> mul_dn(const mat3<T>& a, const mat3<T>& b) { mat3<T> c; gemm<3, 1, 0, 0>(c, a, b); return c; }
// acc += a * b, a * b^dag, a^dag * b
template <typename T>
MAG_HD void mul_acc(mat3<T>& acc, const mat3<T>& a, const mat3<T>& b) { gemm<3, 0, 0, 1>(acc, a, b); }
template <typename T>
MAG_HD void mul_nd_acc(mat3<T>& acc, const mat3<T>& a, const mat3<T>& b) { gemm<3, 0, 1, 1>(acc, a, b); }
template <typename T>
MAG_HD void mul_dn_acc(mat3<T>& acc, const mat3<T>& a, const mat3<T>& b) { gemm<3, 1, 0, 1>(acc, a, b); }
// acc -= a * b
template <typename T>
MAG_HD void mul_sub(mat3<T>& acc, const mat3<T>& a, const mat3<T>& b) { gemm<3, 0, 0, -1>(acc, a, b); }

// ------------------------------------------------ special-unitary products
// A product of SU(3) matrices is in SU(3), so its third row is conj(row0 x
// row1): two rows cost 18 complex multiply-adds instead of 27, and only rows
// 0, 1 of the left factor are read.
template <typename T>
MAG_HD cplx<T> cross_conj(cplx<T> a, cplx<T> b, cplx<T> c, cplx<T> d) {  // conj(a b - c d)
    cplx<T> s;
    s.re = a.re * b.re;
    s.re = fmaT(-a.im, b.im, s.re);
    s.re = fmaT(-c.re, d.re, s.re);
    s.re = fmaT(c.im, d.im, s.re);
    s.im = c.re * d.im;
    s.im = fmaT(c.im, d.re, s.im);
    s.im = fmaT(-a.re, b.im, s.im);
    s.im = fmaT(-a.im, b.re, s.im);
    return s;
}
template <typename T>
MAG_HD void reconstruct_row2(mat3<T>& m) {
    m.e[2][0] = cross_conj(m.e[0][1], m.e[1][2], m.e[0][2], m.e[1][1]);
    m.e[2][1] = cross_conj(m.e[0][2], m.e[1][0], m.e[0][0], m.e[1][2]);
    m.e[2][2] = cross_conj(m.e[0][0], m.e[1][1], m.e[0][1], m.e[1][0]);
}
// rows 0, 1 of a * b, a * b^dag, a^dag * b (row 2 of the result left unset)
template <typename T>
MAG_HD mat3<T> mul_2r(const mat3<T>& a, const mat3<T>& b) { mat3<T> c; gemm<2, 0, 0, 0>(c, a, b); return c; }
template <typename T>
MAG_HD mat3<T> mul_nd_2r(const mat3<T>& a, const mat3<T>& b) { mat3<T> c; gemm<2, 0, 1, 0>(c, a, b); return c; }
template <typename T>
MAG_HD mat3<T> mul_dn_2r(const mat3<T>& a, const mat3<T>& b) { mat3<T> c; gemm<2, 1, 0, 0>(c, a, b); return c; }
// full SU(3) products through two rows + reconstruction
template <typename T>
MAG_HD mat3<T> mul_su3(const mat3<T>& a, const mat3<T>& b) {
    mat3<T> c = mul_2r(a, b);
    reconstruct_row2(c);
    return c;
}
template <typename T>
MAG_HD mat3<T> mul_nd_su3(const mat3<T>& a, const mat3<T>& b) {
    mat3<T> c = mul_nd_2r(a, b);
    reconstruct_row2(c);
    return c;
}
template <typename T>
MAG_HD mat3<T> mul_dn_su3(const mat3<T>& a, const mat3<T>& b) {
    mat3<T> c = mul_dn_2r(a, b);
    reconstruct_row2(c);
    return c;
}

template <typename T>
MAG_HD mat3<T> adj(const mat3<T>& a) {
    mat3<T> c;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) c.e[i][j] = conj(a.e[j][i]);
    return c;
}
template <typename T>
MAG_HD void add_to(mat3<T>& a, const mat3<T>& b) {
#ifdef MAG_F32X2
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) a.e[i][j] = f2::un(__fadd2_rn(f2::nat(a.e[i][j]), f2::nat(b.e[i][j])));
        return;
    }
#endif
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a.e[i][j] = a.e[i][j] + b.e[i][j];
}
template <typename T>
MAG_HD void sub_from(mat3<T>& a, const mat3<T>& b) {
#ifdef MAG_F32X2
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                a.e[i][j] = f2::un(f2::fma2(f2::bc(-1.f), f2::nat(b.e[i][j]), f2::nat(a.e[i][j])));
        return;
    }
#endif
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a.e[i][j] = a.e[i][j] - b.e[i][j];
}
// a += s * b
template <typename T>
MAG_HD void axpy(mat3<T>& a, T s, const mat3<T>& b) {
#ifdef MAG_F32X2
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) a.e[i][j] = f2::un(f2::fma2(f2::bc(s), f2::nat(b.e[i][j]), f2::nat(a.e[i][j])));
        return;
    }
#endif
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            a.e[i][j].re += s * b.e[i][j].re;
            a.e[i][j].im += s * b.e[i][j].im;
        }
}
// a += z * b (complex scalar)
template <typename T>
MAG_HD void caxpy(mat3<T>& a, cplx<T> z, const mat3<T>& b) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) cmac<false, false, false>(a.e[i][j], z, b.e[i][j]);
}
template <typename T>
MAG_HD mat3<T> scaled(const mat3<T>& a, T s) {
    mat3<T> c;
#ifdef MAG_F32X2
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) c.e[i][j] = f2::un(f2::mul2(f2::bc(s), f2::nat(a.e[i][j])));
        return c;
    }
#endif
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) c.e[i][j] = a.e[i][j] * s;
    return c;
}
// i * s * a
template <typename T>
MAG_HD mat3<T> times_i(const mat3<T>& a, T s) {
    mat3<T> c;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) c.e[i][j] = mk(-s * a.e[i][j].im, s * a.e[i][j].re);
    return c;
}
template <typename T>
MAG_HD T retr(const mat3<T>& a) { return a.e[0][0].re + a.e[1][1].re + a.e[2][2].re; }
// Re Tr(a * b) without forming the product
template <typename T>
MAG_HD T retr_mul(const mat3<T>& a, const mat3<T>& b) {
    T s = T(0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            s = fmaT(a.e[i][k].re, b.e[k][i].re, s);
            s = fmaT(-a.e[i][k].im, b.e[k][i].im, s);
        }
    return s;
}
// Re Tr(a * b^dag) = sum_ij Re(a_ij conj(b_ij)) without forming the product
template <typename T>
MAG_HD T retr_mul_nd(const mat3<T>& a, const mat3<T>& b) {
    T s = T(0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            s = fmaT(a.e[i][j].re, b.e[i][j].re, s);
            s = fmaT(a.e[i][j].im, b.e[i][j].im, s);
        }
    return s;
}
// Tr(a * b)
template <typename T>
MAG_HD cplx<T> tr_mul(const mat3<T>& a, const mat3<T>& b) {
    cplx<T> s = mk<T>(0, 0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) cmac<false, false, false>(s, a.e[i][k], b.e[k][i]);
    return s;
}
template <typename T, typename S>
MAG_HD mat3<T> convert(const mat3<S>& a) {
    mat3<T> c;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) c.e[i][j] = mk<T>((T)a.e[i][j].re, (T)a.e[i][j].im);
    return c;
}

// ---------------------------------------------------------- compact Hermitian
template <typename T>
MAG_HD mat3<T> expand(const herm8<T>& q) {
    mat3<T> m;
    m.e[0][0] = mk<T>(q.h[0], 0);
    m.e[1][1] = mk<T>(q.h[1], 0);
    m.e[2][2] = mk<T>(-q.h[0] - q.h[1], 0);
    m.e[0][1] = mk<T>(q.h[2], q.h[3]);
    m.e[1][0] = mk<T>(q.h[2], -q.h[3]);
    m.e[0][2] = mk<T>(q.h[4], q.h[5]);
    m.e[2][0] = mk<T>(q.h[4], -q.h[5]);
    m.e[1][2] = mk<T>(q.h[6], q.h[7]);
    m.e[2][1] = mk<T>(q.h[6], -q.h[7]);
    return m;
}
// compact of a matrix that is Hermitian traceless by construction (upper triangle read)
template <typename T>
MAG_HD herm8<T> compact(const mat3<T>& m) {
    herm8<T> q;
    q.h[0] = m.e[0][0].re; q.h[1] = m.e[1][1].re;
    q.h[2] = m.e[0][1].re; q.h[3] = m.e[0][1].im;
    q.h[4] = m.e[0][2].re; q.h[5] = m.e[0][2].im;
    q.h[6] = m.e[1][2].re; q.h[7] = m.e[1][2].im;
    return q;
}
template <typename T>
MAG_HD herm8<T> herm_zero() { herm8<T> q; for (int k = 0; k < 8; k++) q.h[k] = T(0); return q; }
template <typename T>
MAG_HD herm8<T> scaled(const herm8<T>& a, T s) { herm8<T> q; for (int k = 0; k < 8; k++) q.h[k] = a.h[k] * s; return q; }

// Products with a Hermitian traceless factor read straight from the compact
// form: its diagonal is real, so an element costs one real-complex and two
// complex-complex products.
//   H = [[h0, z01, z02], [z01*, h1, z12], [z02*, z12*, -h0-h1]]
template <typename T>
MAG_HD void herm_rows(const herm8<T>& q, cplx<T> H[3][3]) {
    H[0][0] = mk<T>(q.h[0], 0);
    H[1][1] = mk<T>(q.h[1], 0);
    H[2][2] = mk<T>(-q.h[0] - q.h[1], 0);
    H[0][1] = mk<T>(q.h[2], q.h[3]);
    H[1][0] = mk<T>(q.h[2], -q.h[3]);
    H[0][2] = mk<T>(q.h[4], q.h[5]);
    H[2][0] = mk<T>(q.h[4], -q.h[5]);
    H[1][2] = mk<T>(q.h[6], q.h[7]);
    H[2][1] = mk<T>(q.h[6], -q.h[7]);
}
// c (=, +=, -=) H op(X)  (SIDE = 0)  or  op(X) H  (SIDE = 1); TX = 1: op(X) = X^dag
template <int SIDE, int TX, int ACC, typename T>
MAG_HD void hgemm(mat3<T>& c, const herm8<T>& q, const mat3<T>& x) {
    cplx<T> H[3][3];
    herm_rows(q, H);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int d = SIDE == 0 ? i : j;  // index of the real diagonal element of H in this sum
            cplx<T> s;
            if (ACC == 0) {
                const cplx<T> xd = TX ? conj(SIDE == 0 ? x.e[j][d] : x.e[d][i]) : (SIDE == 0 ? x.e[d][j] : x.e[i][d]);
                s = mk(H[d][d].re * xd.re, H[d][d].re * xd.im);
            } else {
                s = c.e[i][j];
                const cplx<T> xd = TX ? conj(SIDE == 0 ? x.e[j][d] : x.e[d][i]) : (SIDE == 0 ? x.e[d][j] : x.e[i][d]);
                const T h = ACC < 0 ? -H[d][d].re : H[d][d].re;
                s.re = fmaT(h, xd.re, s.re);
                s.im = fmaT(h, xd.im, s.im);
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                if (k == d) continue;
                if (SIDE == 0) {  // H[i][k] op(X)[k][j]
                    const cplx<T> xk = TX ? x.e[j][k] : x.e[k][j];
                    cmac<false, TX != 0, (ACC < 0)>(s, H[i][k], xk);
                } else {          // op(X)[i][k] H[k][j]
                    const cplx<T> xk = TX ? x.e[k][i] : x.e[i][k];
                    cmac<TX != 0, false, (ACC < 0)>(s, xk, H[k][j]);
                }
            }
            c.e[i][j] = s;
        }
}
// H X, H X^dag, X H, X^dag H and their accumulating forms
template <typename T>
MAG_HD mat3<T> mul_hm(const herm8<T>& q, const mat3<T>& x) { mat3<T> c; hgemm<0, 0, 0>(c, q, x); return c; }
template <typename T>
MAG_HD mat3<T> mul_hm_nd(const herm8<T>& q, const mat3<T>& x) { mat3<T> c; hgemm<0, 1, 0>(c, q, x); return c; }
template <typename T>
MAG_HD mat3<T> mul_mh(const mat3<T>& x, const herm8<T>& q) { mat3<T> c; hgemm<1, 0, 0>(c, q, x); return c; }
template <typename T>
MAG_HD mat3<T> mul_dn_mh(const mat3<T>& x, const herm8<T>& q) { mat3<T> c; hgemm<1, 1, 0>(c, q, x); return c; }
template <typename T>
MAG_HD void mul_hm_acc(mat3<T>& c, const herm8<T>& q, const mat3<T>& x) { hgemm<0, 0, 1>(c, q, x); }
template <typename T>
MAG_HD void mul_hm_sub(mat3<T>& c, const herm8<T>& q, const mat3<T>& x) { hgemm<0, 0, -1>(c, q, x); }
template <typename T>
MAG_HD void mul_hm_nd_sub(mat3<T>& c, const herm8<T>& q, const mat3<T>& x) { hgemm<0, 1, -1>(c, q, x); }
template <typename T>
MAG_HD void mul_mh_acc(mat3<T>& c, const mat3<T>& x, const herm8<T>& q) { hgemm<1, 0, 1>(c, q, x); }

// F = i s TA(M),  TA(M) = 1/2 (M - M^dag) - 1/6 Tr(M - M^dag)  (cps TrLessAntiHermMatrix)
template <typename T>
MAG_HD herm8<T> i_times_ta(const mat3<T>& m, T s) {
    const T t = (m.e[0][0].im + m.e[1][1].im + m.e[2][2].im) / T(3);
    herm8<T> q;
    q.h[0] = -s * (m.e[0][0].im - t);
    q.h[1] = -s * (m.e[1][1].im - t);
    // off-diagonal TA_ij = (1/2 (Re M_ij - Re M_ji), 1/2 (Im M_ij + Im M_ji)); times i s
    q.h[2] = -s * (T(0.5) * (m.e[0][1].im + m.e[1][0].im));
    q.h[3] = s * (T(0.5) * (m.e[0][1].re - m.e[1][0].re));
    q.h[4] = -s * (T(0.5) * (m.e[0][2].im + m.e[2][0].im));
    q.h[5] = s * (T(0.5) * (m.e[0][2].re - m.e[2][0].re));
    q.h[6] = -s * (T(0.5) * (m.e[1][2].im + m.e[2][1].im));
    q.h[7] = s * (T(0.5) * (m.e[1][2].re - m.e[2][1].re));
    return q;
}
// Lambda = 1/2 (G + G^dag) - 1/6 Tr(G + G^dag)  (field-multi.h:41-45)
template <typename T>
MAG_HD herm8<T> herm_traceless(const mat3<T>& g) {
    const T t = (g.e[0][0].re + g.e[1][1].re + g.e[2][2].re) / T(3);
    herm8<T> q;
    q.h[0] = g.e[0][0].re - t;
    q.h[1] = g.e[1][1].re - t;
    q.h[2] = T(0.5) * (g.e[0][1].re + g.e[1][0].re);
    q.h[3] = T(0.5) * (g.e[0][1].im - g.e[1][0].im);
    q.h[4] = T(0.5) * (g.e[0][2].re + g.e[2][0].re);
    q.h[5] = T(0.5) * (g.e[0][2].im - g.e[2][0].im);
    q.h[6] = T(0.5) * (g.e[1][2].re + g.e[2][1].re);
    q.h[7] = T(0.5) * (g.e[1][2].im - g.e[2][1].im);
    return q;
}
// Re Tr(H^2) of a compact Hermitian traceless matrix
template <typename T>
MAG_HD T retr_sq(const herm8<T>& q) {
    const T h22 = -q.h[0] - q.h[1];
    return q.h[0] * q.h[0] + q.h[1] * q.h[1] + h22 * h22 +
           T(2) * (q.h[2] * q.h[2] + q.h[3] * q.h[3] + q.h[4] * q.h[4] + q.h[5] * q.h[5] + q.h[6] * q.h[6] +
                   q.h[7] * q.h[7]);
}

// CPS Matrix::Unitarize: normalise row 0, orthogonalise row 1 to it and
// normalise, row 2 = conj(row0 x row1).
template <typename T>
MAG_HD void unitarize(mat3<T>& m) {
    T n0 = T(0);
#pragma unroll
    for (int k = 0; k < 3; k++) n0 += m.e[0][k].re * m.e[0][k].re + m.e[0][k].im * m.e[0][k].im;
    n0 = T(1) / sqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; k++) m.e[0][k] = m.e[0][k] * n0;
    cplx<T> c = mk<T>(0, 0);
#pragma unroll
    for (int k = 0; k < 3; k++) c = c + conj(m.e[0][k]) * m.e[1][k];
#pragma unroll
    for (int k = 0; k < 3; k++) m.e[1][k] = m.e[1][k] - c * m.e[0][k];
    T n1 = T(0);
#pragma unroll
    for (int k = 0; k < 3; k++) n1 += m.e[1][k].re * m.e[1][k].re + m.e[1][k].im * m.e[1][k].im;
    n1 = T(1) / sqrt(n1);
#pragma unroll
    for (int k = 0; k < 3; k++) m.e[1][k] = m.e[1][k] * n1;
    m.e[2][0] = conj(m.e[0][1] * m.e[1][2] - m.e[0][2] * m.e[1][1]);
    m.e[2][1] = conj(m.e[0][2] * m.e[1][0] - m.e[0][0] * m.e[1][2]);
    m.e[2][2] = conj(m.e[0][0] * m.e[1][1] - m.e[0][1] * m.e[1][0]);
}

// -------------------------------------------------- Cayley-Hamilton exp(iQ)
// Scalar part of hep-lat/0311018 as written in field-hmc.h:88-115 (expiQ) and
// field-multi.h:92-168 (DexpiQ / compute_Lambda).  Always evaluated in double:
// the FP32 kernels call it too, because the f_j and b_ij formulas cancel
// catastrophically in single precision.
struct ch_coef {
    int trivial;  // c1 == 0: expiQ = 1, derivative terms = 0
    double f0r, f0i, f1r, f1i, f2r, f2i;
    double b10r, b10i, b11r, b11i, b12r, b12i;
    double b20r, b20i, b21r, b21i, b22r, b22i;
};

// c0 = Re Tr(Q^3)/3, c1 = Re Tr(Q^2)/2 as supplied by the caller.
MAG_HD void sincos_hd(double x, double& s, double& c) {
#if defined(__CUDA_ARCH__)
    sincos(x, &s, &c);
#else
    s = sin(x);
    c = cos(x);
#endif
}

template <bool WITH_B>
MAG_HD ch_coef ch_coefficients(double c0, double c1) {
    ch_coef r;
    r.trivial = 0;
    bool reflect = false;
    if (c0 < 0.0) { c0 = -c0; reflect = true; }
    if (c1 == 0.0) {
        r.trivial = 1;
        r.f0r = 1.0; r.f0i = r.f1r = r.f1i = r.f2r = r.f2i = 0.0;
        r.b10r = r.b10i = r.b11r = r.b11i = r.b12r = r.b12i = 0.0;
        r.b20r = r.b20i = r.b21r = r.b21i = r.b22r = r.b22i = 0.0;
        return r;
    }
    // The same quantities as the reference (field-hmc.h:90-110), evaluated with
    // fewer library calls: (c1/3)^1.5 = t sqrt(t), sqrt(c1) = sqrt(3) sqrt(c1/3),
    // sine and cosine of one argument from one sincos, cos 2u and sin 2u by the
    // double-angle formulas, divisions by den as products with 1/den.
    const double t3 = c1 / 3.0, st3 = sqrt(t3);
    const double c0m = 2.0 * t3 * st3;
    double ratio = c0 / c0m;
    if (ratio > 1.0) ratio = 1.0;  // rounding guard (reference would return NaN)
    const double theta = acos(ratio);
    double sth, cth;
    sincos_hd(theta / 3.0, sth, cth);
    const double u = st3 * cth;
    const double w = 1.7320508075688772 * st3 * sth;  // sqrt(c1) sin(theta / 3)
    const double ww = w * w, uu = u * u;
    double sw, cw;
    sincos_hd(w, sw, cw);
    double xi0, xi1 = 0.0;
    if (ww < 0.05 * 0.05) {
        xi0 = 1. - ww / 6. * (1. - ww / 20. * (1. - ww / 42.));
        if (WITH_B) xi1 = -1. / 2. * (1. - ww / 12. * (1. - ww / 30.)) + 1. / 6. * (1. - ww / 20. * (1. - ww / 42.));
    } else {
        const double iw = 1.0 / w;
        xi0 = sw * iw;
        if (WITH_B) xi1 = (cw - xi0) * iw * iw;  // cos(w)/w^2 - sin(w)/w^3
    }
    double su, cu;
    sincos_hd(u, su, cu);
    const double c2u = (cu - su) * (cu + su), s2u = 2.0 * su * cu;
    // e2u = exp(2iu), emu = exp(-iu)
    // h0 = (u^2-w^2) e2u + emu (8u^2 cos w + i 2u(3u^2+w^2) xi0)
    const double a0r = 8. * uu * cw, a0i = 2. * u * (3. * uu + ww) * xi0;
    const double h0r = (uu - ww) * c2u + (cu * a0r + su * a0i);
    const double h0i = (uu - ww) * s2u + (cu * a0i - su * a0r);
    // h1 = 2u e2u - emu (2u cos w - i (3u^2-w^2) xi0)
    const double a1r = 2. * u * cw, a1i = -(3. * uu - ww) * xi0;
    const double h1r = 2. * u * c2u - (cu * a1r + su * a1i);
    const double h1i = 2. * u * s2u - (cu * a1i - su * a1r);
    // h2 = e2u - emu (cos w + i 3u xi0)
    const double a2r = cw, a2i = 3. * u * xi0;
    const double h2r = c2u - (cu * a2r + su * a2i);
    const double h2i = s2u - (cu * a2i - su * a2r);
    const double den = 9. * uu - ww, iden = 1.0 / den;
    double f0r = h0r * iden, f0i = h0i * iden, f1r = h1r * iden, f1i = h1i * iden, f2r = h2r * iden,
           f2i = h2i * iden;
    if (WITH_B) {
        // complex helpers in (re, im) pairs
        // r01 = 2(u + i(u^2-w^2)) e2u + 2 emu (4u(2 - iu) cos w + i xi0 (9u^2 + w^2 - iu(3u^2+w^2)))
        double tr_, ti_;
        // term A = 2(u + i(uu-ww)) * e2u
        const double Ar = 2. * (u * c2u - (uu - ww) * s2u), Ai = 2. * (u * s2u + (uu - ww) * c2u);
        // inner B = 4u(2 - iu) cw + i xi0 (9uu + ww - iu(3uu+ww))
        //         = (8u cw + xi0 u (3uu+ww)) + i(-4uu cw + xi0 (9uu + ww))
        const double Br = 8. * u * cw + xi0 * u * (3. * uu + ww), Bi = -4. * uu * cw + xi0 * (9. * uu + ww);
        tr_ = 2. * (cu * Br + su * Bi); ti_ = 2. * (cu * Bi - su * Br);
        const double r01r = Ar + tr_, r01i = Ai + ti_;
        // r11 = 2(1 + 2iu) e2u + emu(-2(1 - iu) cw + i xi0 (6u + i(ww - 3uu)))
        const double Cr = 2. * (c2u - 2. * u * s2u), Ci = 2. * (s2u + 2. * u * c2u);
        // inner D = -2cw + 2iu cw + i 6u xi0 - xi0 (ww - 3uu)
        const double Dr = -2. * cw - xi0 * (ww - 3. * uu), Di = 2. * u * cw + 6. * u * xi0;
        const double r11r = Cr + (cu * Dr + su * Di), r11i = Ci + (cu * Di - su * Dr);
        // r21 = 2i e2u + i emu (cw - 3 xi0 (1 - iu))
        //   inner E = (cw - 3xi0) + i 3u xi0 ; i*emu*E
        const double Er = cw - 3. * xi0, Ei = 3. * u * xi0;
        const double eEr = cu * Er + su * Ei, eEi = cu * Ei - su * Er;
        const double r21r = -2. * s2u - eEi, r21i = 2. * c2u + eEr;
        // r02 = -2 e2u + 2iu emu (cw + (1 + 4iu) xi0 + 3uu xi1)
        const double Fr = cw + xi0 + 3. * uu * xi1, Fi = 4. * u * xi0;
        const double eFr = cu * Fr + su * Fi, eFi = cu * Fi - su * Fr;
        const double r02r = -2. * c2u - 2. * u * eFi, r02i = -2. * s2u + 2. * u * eFr;
        // r12 = -i emu (cw + (1 + 2iu) xi0 - 3uu xi1)
        const double Gr = cw + xi0 - 3. * uu * xi1, Gi = 2. * u * xi0;
        const double eGr = cu * Gr + su * Gi, eGi = cu * Gi - su * Gr;
        const double r12r = eGi, r12i = -eGr;
        // r22 = emu (xi0 - 3iu xi1)
        const double Hr = xi0, Hi = -3. * u * xi1;
        const double r22r = cu * Hr + su * Hi, r22i = cu * Hi - su * Hr;
        const double ibden = 0.5 * iden * iden;  // 1 / (2 den^2)
        const double k1 = 3. * uu - ww, k2 = 2. * (15. * uu + ww);
        r.b10r = (2. * u * r01r + k1 * r02r - k2 * f0r) * ibden;
        r.b10i = (2. * u * r01i + k1 * r02i - k2 * f0i) * ibden;
        r.b11r = (2. * u * r11r + k1 * r12r - k2 * f1r) * ibden;
        r.b11i = (2. * u * r11i + k1 * r12i - k2 * f1i) * ibden;
        r.b12r = (2. * u * r21r + k1 * r22r - k2 * f2r) * ibden;
        r.b12i = (2. * u * r21i + k1 * r22i - k2 * f2i) * ibden;
        r.b20r = (r01r - 3. * u * r02r - 24. * u * f0r) * ibden;
        r.b20i = (r01i - 3. * u * r02i - 24. * u * f0i) * ibden;
        r.b21r = (r11r - 3. * u * r12r - 24. * u * f1r) * ibden;
        r.b21i = (r11i - 3. * u * r12i - 24. * u * f1i) * ibden;
        r.b22r = (r21r - 3. * u * r22r - 24. * u * f2r) * ibden;
        r.b22i = (r21i - 3. * u * r22i - 24. * u * f2i) * ibden;
        if (reflect) {
            r.b10i = -r.b10i;                 // conj
            r.b11r = -r.b11r;                 // -conj
            r.b12i = -r.b12i;                 // conj
            r.b20r = -r.b20r;                 // -conj
            r.b21i = -r.b21i;                 // conj
            r.b22r = -r.b22r;                 // -conj
        }
    } else {
        r.b10r = r.b10i = r.b11r = r.b11i = r.b12r = r.b12i = 0.0;
        r.b20r = r.b20i = r.b21r = r.b21i = r.b22r = r.b22i = 0.0;
    }
    if (reflect) {
        f0i = -f0i;    // conj
        f1r = -f1r;    // -conj
        f2i = -f2i;    // conj
    }
    r.f0r = f0r; r.f0i = f0i; r.f1r = f1r; r.f1i = f1i; r.f2r = f2r; r.f2i = f2i;
    return r;
}

// Single-precision Cayley-Hamilton coefficients by the power series of exp(iQ)
// in the invariants.  For traceless Q, Q^3 = c1 Q + c0 with c0 = det Q =
// Tr(Q^3)/3 and c1 = Tr(Q^2)/2, so Q^n = a_n + b_n Q + d_n Q^2 with
//   a_{n+1} = c0 d_n,  b_{n+1} = a_n + c1 d_n,  d_{n+1} = b_n,
// and f_j = sum_n i^n/n! (a_n, b_n, d_n)_j.  The derivative coefficients of
// hep-lat/0311018 are b_1j = df_j/dc1 and b_2j = df_j/dc0 (dc1 = Tr(Q dQ),
// dc0 = Tr(Q^2 dQ)), carried by differentiating the recurrence.  All terms
// are real times a power of i, so nothing cancels beyond the alternating
// series itself; with |eigenvalue| <= q = sqrt(4 c1 / 3) the sum stops when
// q^n / n! < 1e-9.  Used by the FP32 kernels; returns false (and the caller
// falls back to the double closed form) when q > 3.
struct ch_coef_f {
    float f0r, f0i, f1r, f1i, f2r, f2i;
    float b10r, b10i, b11r, b11i, b12r, b12i;
    float b20r, b20i, b21r, b21i, b22r, b22i;
};

template <bool WITH_B>
MAG_HD bool ch_series(float c0, float c1, ch_coef_f& r) {
    const float q2 = (4.f / 3.f) * c1;
    if (q2 > 9.f) return false;
    float a = 1.f, b = 0.f, d = 0.f;                       // Q^n coefficients
    float a0 = 0.f, b0 = 0.f, d0 = 0.f, a1 = 0.f, b1 = 0.f, d1 = 0.f;  // d/dc0, d/dc1
    // f_j and the b coefficients, real and imaginary parts apart (n = 0 term: f_0 = 1)
    float Fr[3] = {1.f, 0.f, 0.f}, Fi[3] = {0.f, 0.f, 0.f};
    float B1r[3] = {0.f, 0.f, 0.f}, B1i[3] = {0.f, 0.f, 0.f};
    float B2r[3] = {0.f, 0.f, 0.f}, B2i[3] = {0.f, 0.f, 0.f};
    float coef = 1.f;    // 1/n!
    float bound = 1.f;   // q^n / n! for q >= 1, q^(n-5) / n! for q < 1: the a_n, b_n, d_n
                         // and their derivatives carry powers of q down to q^(n-5)
    const float q = sqrtf(q2);
    const bool qbig = q >= 1.f;
    // one term: advance Q^{n-1} -> Q^n (and the derivatives), add i^n/n! times it; the loop
    // below is unrolled, so n and 1/n are compile-time constants (no division is executed)
    auto term = [&](int n, bool odd) {
        const float na = c0 * d, nb = a + c1 * d, nd = b;
        if (WITH_B) {
            const float na0 = d + c0 * d0, nb0 = a0 + c1 * d0, nd0 = b0;
            const float na1 = c0 * d1, nb1 = a1 + d + c1 * d1, nd1 = b1;
            a0 = na0; b0 = nb0; d0 = nd0;
            a1 = na1; b1 = nb1; d1 = nd1;
        }
        a = na; b = nb; d = nd;
        const float inv = 1.f / (float)n;
        coef *= inv;
        bound *= (qbig || n > 5 ? q : 1.f) * inv;
        // i^n/n!: real for even n (sign (-1)^{n/2}), imaginary for odd n (sign (-1)^{(n-1)/2})
        const float sgn = ((n >> 1) & 1) ? -coef : coef;
        float* F = odd ? Fi : Fr;
        F[0] = fmaf(sgn, a, F[0]);
        F[1] = fmaf(sgn, b, F[1]);
        F[2] = fmaf(sgn, d, F[2]);
        if (WITH_B) {
            float* P = odd ? B1i : B1r;
            float* R = odd ? B2i : B2r;
            P[0] = fmaf(sgn, a1, P[0]); P[1] = fmaf(sgn, b1, P[1]); P[2] = fmaf(sgn, d1, P[2]);
            R[0] = fmaf(sgn, a0, R[0]); R[1] = fmaf(sgn, b0, R[1]); R[2] = fmaf(sgn, d0, R[2]);
        }
    };
    // terms in pairs (odd, even) so that the real / imaginary choice is known at compile time
#pragma unroll
    for (int n = 1; n < 40; n += 2) {
        term(n, true);
        term(n + 1, false);
        if (n + 1 > 5 && bound < 1e-9f) break;
    }
    r.f0r = Fr[0]; r.f0i = Fi[0]; r.f1r = Fr[1]; r.f1i = Fi[1]; r.f2r = Fr[2]; r.f2i = Fi[2];
    r.b10r = B1r[0]; r.b10i = B1i[0]; r.b11r = B1r[1]; r.b11i = B1i[1]; r.b12r = B1r[2]; r.b12i = B1i[2];
    r.b20r = B2r[0]; r.b20i = B2i[0]; r.b21r = B2r[1]; r.b21i = B2i[1]; r.b22r = B2r[2]; r.b22i = B2i[2];
    return true;
}

// the same coefficients from the double closed form
MAG_HD ch_coef_f ch_to_float(const ch_coef& c) {
    ch_coef_f r;
    r.f0r = (float)c.f0r; r.f0i = (float)c.f0i; r.f1r = (float)c.f1r; r.f1i = (float)c.f1i;
    r.f2r = (float)c.f2r; r.f2i = (float)c.f2i;
    r.b10r = (float)c.b10r; r.b10i = (float)c.b10i; r.b11r = (float)c.b11r; r.b11i = (float)c.b11i;
    r.b12r = (float)c.b12r; r.b12i = (float)c.b12i;
    r.b20r = (float)c.b20r; r.b20i = (float)c.b20i; r.b21r = (float)c.b21r; r.b21i = (float)c.b21i;
    r.b22r = (float)c.b22r; r.b22i = (float)c.b22i;
    return r;
}

// exp(iQ)'s coefficients f_j alone, in double, by the same series as
// ch_series: f_j = sum_n i^n/n! (a_n, b_n, d_n)_j with Q^n = a_n + b_n Q + d_n Q^2.
// The terms are unrolled in (odd, even) pairs with 1/n folded to constants;
// with q = sqrt(4 c1 / 3) >= every eigenvalue modulus, a_n, b_n, d_n are
// bounded by q^n (q >= 1) or q^(n-2) (q < 1), so the sum stops once
// q^n / n! (or q^(n-2) / n!) falls below 1e-17: about 10 terms for the
// exponents of a link update (q ~ 0.1), 16 for a stout level (q ~ 0.5).
// No transcendental function is evaluated.  exp(iQ) from these f_j agrees
// with exp(iQ) from the closed form to rounding (a long-double Taylor check:
// <= 3e-15 for Q entries of scale 1e-4 to 2, against the closed form's
// <= 6e-16 to 3e-15): the closed form's own f_j lose accuracy at small Q
// (|df| ~ 1e-12 at scale 0.01), but those errors reach exp(iQ) multiplied by
// Q and Q^2.  The derivative coefficients b_ij of compute_Lambda have no such
// damping, which is why the FP64 Lambda keeps the reference's closed form
// (same numbers as the reference, errors included).  Returns false for q > 3.
MAG_HD bool ch_series_exp_d(double c0, double c1, double f[6]) {
    const double q2 = (4.0 / 3.0) * c1;
    if (q2 > 9.0) return false;
    const double q = sqrt(q2);
    const bool qbig = q >= 1.0;
    double a = 1.0, b = 0.0, d = 0.0;
    double f0r = 1.0, f1r = 0.0, f2r = 0.0, f0i = 0.0, f1i = 0.0, f2i = 0.0;
    double coef = 1.0, bound = 1.0;
#pragma unroll
    for (int n = 1; n < 40; n += 2) {
        {  // odd term: i^n = (-1)^((n-1)/2) i
            const double na = c0 * d, nb = fmaT(c1, d, a), nd = b;
            a = na; b = nb; d = nd;
            coef *= 1.0 / n;
            bound *= (qbig || n > 2 ? q : 1.0) * (1.0 / n);
            const double sg = ((n >> 1) & 1) ? -coef : coef;
            f0i = fmaT(sg, a, f0i);
            f1i = fmaT(sg, b, f1i);
            f2i = fmaT(sg, d, f2i);
        }
        {  // even term n + 1: i^(n+1) = (-1)^((n+1)/2)
            const int m = n + 1;
            const double na = c0 * d, nb = fmaT(c1, d, a), nd = b;
            a = na; b = nb; d = nd;
            coef *= 1.0 / m;
            bound *= (qbig || m > 2 ? q : 1.0) * (1.0 / m);
            const double sg = ((m >> 1) & 1) ? -coef : coef;
            f0r = fmaT(sg, a, f0r);
            f1r = fmaT(sg, b, f1r);
            f2r = fmaT(sg, d, f2r);
        }
        if (n + 1 >= 4 && bound < 1e-17) break;
    }
    f[0] = f0r; f[1] = f0i; f[2] = f1r; f[3] = f1i; f[4] = f2r; f[5] = f2i;
    return true;
}

// Q^2 of a compact Hermitian traceless matrix (Hermitian result)
template <typename T>
MAG_HD mat3<T> herm_square(const herm8<T>& q) {
    const mat3<T> Q = expand(q);
    return mul(Q, Q);
}

// c0 = Re Tr(Q^3)/3 and c1 = Re Tr(Q^2)/2 in double (as field-hmc.h:88-94)
template <typename T>
MAG_HD void ch_invariants(const mat3<T>& Q, const mat3<T>& QQ, double& c0, double& c1) {
    double t3 = 0.0, t2 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        t2 += (double)QQ.e[i][i].re;
#pragma unroll
        for (int k = 0; k < 3; k++)
            t3 += (double)QQ.e[i][k].re * (double)Q.e[k][i].re - (double)QQ.e[i][k].im * (double)Q.e[k][i].im;
    }
    c0 = t3 / 3.0;
    c1 = t2 / 2.0;
}

// single-precision invariants c0 = Re Tr(Q^3)/3, c1 = Re Tr(Q^2)/2
MAG_HD void ch_invariants_f(const mat3<float>& Q, const mat3<float>& QQ, float& c0, float& c1) {
    float t3 = 0.f;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) t3 += QQ.e[i][k].re * Q.e[k][i].re - QQ.e[i][k].im * Q.e[k][i].im;
    c0 = t3 * (1.f / 3.f);
    c1 = 0.5f * (QQ.e[0][0].re + QQ.e[1][1].re + QQ.e[2][2].re);
}

// Cayley-Hamilton coefficients for a matrix of precision T: the reference's
// closed form in double for T = double; the power series for T = float (the
// closed form in double when the series would be too long).  trivial: c1 = 0,
// where the reference returns exp(iQ) = 1 and Lambda = 0.
template <typename T, bool WITH_B>
MAG_HD bool ch_for(const mat3<T>& Q, const mat3<T>& QQ, ch_coef_f& cf) {
    if constexpr (sizeof(T) == 4) {
        float c0, c1;
        ch_invariants_f(Q, QQ, c0, c1);
        if (c1 == 0.f) return false;
        if (ch_series<WITH_B>(c0, c1, cf)) return true;
    }
    double c0, c1;
    ch_invariants(Q, QQ, c0, c1);
    const ch_coef c = ch_coefficients<WITH_B>(c0, c1);
    if (c.trivial) return false;
    cf = ch_to_float(c);
    return true;
}

// exp(iQ) = f0 + f1 Q + f2 Q^2 (field-hmc.h:82-123)
template <typename T>
MAG_HD mat3<T> expiQ(const herm8<T>& q) {
    const mat3<T> Q = expand(q);
    const mat3<T> QQ = mul_hm(q, Q);
    cplx<T> f0, f1, f2;
    if constexpr (sizeof(T) == 4) {
        ch_coef_f c;
        if (!ch_for<T, false>(Q, QQ, c)) return unit_mat<T>();
        f0 = mk(c.f0r, c.f0i);
        f1 = mk(c.f1r, c.f1i);
        f2 = mk(c.f2r, c.f2i);
    } else {
        double c0, c1;
        ch_invariants(Q, QQ, c0, c1);
        if (c1 == 0.0) return unit_mat<T>();  // the reference's c1 = 0 branch (field-hmc.h:95)
        double fs[6];
        if (ch_series_exp_d(c0, c1, fs)) {
            f0 = mk<T>(fs[0], fs[1]);
            f1 = mk<T>(fs[2], fs[3]);
            f2 = mk<T>(fs[4], fs[5]);
        } else {
            const ch_coef c = ch_coefficients<false>(c0, c1);
            f0 = mk<T>((T)c.f0r, (T)c.f0i);
            f1 = mk<T>((T)c.f1r, (T)c.f1i);
            f2 = mk<T>((T)c.f2r, (T)c.f2i);
        }
    }
    mat3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cplx<T> e = cmul<false, false>(f1, Q.e[i][j]);
            cmac<false, false, false>(e, f2, QQ.e[i][j]);
            r.e[i][j] = e;
        }
#pragma unroll
    for (int i = 0; i < 3; i++) r.e[i][i] = r.e[i][i] + f0;
    return r;
}

}  // namespace magb
