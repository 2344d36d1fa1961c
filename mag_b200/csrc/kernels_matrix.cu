// kernels_matrix.cu -- the single-matrix operators of the reference, batched: expiQ
// (field-hmc.h:82-123), DexpiQ (field-multi.h:90-178) and compute_Lambda
// (field-multi.h:180-269) over n matrices in the
// reference's memory image (3x3 complex doubles, row-major re/im).  They run the device
// code of the link update and of the stout chain rule (su3.cuh expiQ, gauge_ops.cuh
// stout_lambda), one thread per matrix.
#include "gauge_ops.cuh"
#include "kernels.h"

namespace magb {

namespace {

constexpr int kMatBlock = 128;

__device__ __forceinline__ mat3<double> load_aos(const double2* p, long i) {
    mat3<double> m;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const double2 v = p[i * 9 + k];
        m.e[k / 3][k % 3] = mk(v.x, v.y);
    }
    return m;
}
__device__ __forceinline__ void store_aos(double2* p, long i, const mat3<double>& m) {
#pragma unroll
    for (int k = 0; k < 9; k++) p[i * 9 + k] = make_double2(m.e[k / 3][k % 3].re, m.e[k / 3][k % 3].im);
}

__global__ void __launch_bounds__(kMatBlock) k_expiq(const double2* q, long n, double2* out) {
    const long i = (long)blockIdx.x * kMatBlock + threadIdx.x;
    if (i >= n) return;
    store_aos(out, i, expiQ(compact(load_aos(q, i))));
}

// d/dt exp(i(Q + t DQ)) at t = 0 by the Cayley-Hamilton coefficients and their derivatives:
//   B1 Tr(Q DQ) + B2 Tr(Q^2 DQ) + f1 DQ + f2 (DQ Q + Q DQ),  B_i = b_i0 + b_i1 Q + b_i2 Q^2;
// zero when c1 = 0, as the reference returns (field-multi.h:100)
__device__ mat3<double> dexpiq(const herm8<double>& q, const mat3<double>& D) {
    const mat3<double> Q = expand(q);
    const mat3<double> QQ = mul_hm(q, Q);
    double c0, c1;
    ch_invariants(Q, QQ, c0, c1);
    const ch_coef c = ch_coefficients<true>(c0, c1);
    mat3<double> r;
    set_zero(r);
    if (c.trivial) return r;
    const cplx<double> t1 = tr_mul(Q, D), t2 = tr_mul(QQ, D);
    cplx<double> a0 = cmul<false, false>(mk(c.b10r, c.b10i), t1);
    cmac<false, false, false>(a0, mk(c.b20r, c.b20i), t2);
    cplx<double> a1 = cmul<false, false>(mk(c.b11r, c.b11i), t1);
    cmac<false, false, false>(a1, mk(c.b21r, c.b21i), t2);
    cplx<double> a2 = cmul<false, false>(mk(c.b12r, c.b12i), t1);
    cmac<false, false, false>(a2, mk(c.b22r, c.b22i), t2);
    mat3<double> DQQD = mul_mh(D, q);  // DQ Q + Q DQ
    mul_hm_acc(DQQD, q, D);
    const cplx<double> f1 = mk(c.f1r, c.f1i), f2 = mk(c.f2r, c.f2i);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cplx<double> e = cmul<false, false>(a1, Q.e[i][j]);
            cmac<false, false, false>(e, a2, QQ.e[i][j]);
            cmac<false, false, false>(e, f1, D.e[i][j]);
            cmac<false, false, false>(e, f2, DQQD.e[i][j]);
            r.e[i][j] = e;
        }
#pragma unroll
    for (int i = 0; i < 3; i++) r.e[i][i] = r.e[i][i] + a0;
    return r;
}

__global__ void __launch_bounds__(kMatBlock) k_dexpiq(const double2* q, const double2* dq, long n, double2* out) {
    const long i = (long)blockIdx.x * kMatBlock + threadIdx.x;
    if (i >= n) return;
    store_aos(out, i, dexpiq(compact(load_aos(q, i)), load_aos(dq, i)));
}

__global__ void __launch_bounds__(kMatBlock) k_compute_lambda(const double2* q, const double2* sigma,
                                                              const double2* u, long n, double2* lam) {
    const long i = (long)blockIdx.x * kMatBlock + threadIdx.x;
    if (i >= n) return;
    herm8<double> l;
    mat3<double> zp;
    stout_lambda(compact(load_aos(q, i)), load_aos(sigma, i), load_aos(u, i), l, zp);
    store_aos(lam, i, expand(l));
}

}  // namespace

void launch_expiq(const double* q, long n, double* out, cudaStream_t s) {
    if (n <= 0) return;
    k_expiq<<<(unsigned)((n + kMatBlock - 1) / kMatBlock), kMatBlock, 0, s>>>(
        reinterpret_cast<const double2*>(q), n, reinterpret_cast<double2*>(out));
}

void launch_dexpiq(const double* q, const double* dq, long n, double* out, cudaStream_t s) {
    if (n <= 0) return;
    k_dexpiq<<<(unsigned)((n + kMatBlock - 1) / kMatBlock), kMatBlock, 0, s>>>(
        reinterpret_cast<const double2*>(q), reinterpret_cast<const double2*>(dq), n,
        reinterpret_cast<double2*>(out));
}

void launch_compute_lambda(const double* q, const double* sigma, const double* u, long n, double* lam,
                           cudaStream_t s) {
    if (n <= 0) return;
    k_compute_lambda<<<(unsigned)((n + kMatBlock - 1) / kMatBlock), kMatBlock, 0, s>>>(
        reinterpret_cast<const double2*>(q), reinterpret_cast<const double2*>(sigma),
        reinterpret_cast<const double2*>(u), n, reinterpret_cast<double2*>(lam));
}

}  // namespace magb
