// kernels_matrix.cu -- the single-matrix operators of the reference, batched: expiQ
// (field-hmc.h:82-123) and compute_Lambda (field-multi.h:180-269) over n matrices in the
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

void launch_compute_lambda(const double* q, const double* sigma, const double* u, long n, double* lam,
                           cudaStream_t s) {
    if (n <= 0) return;
    k_compute_lambda<<<(unsigned)((n + kMatBlock - 1) / kMatBlock), kMatBlock, 0, s>>>(
        reinterpret_cast<const double2*>(q), reinterpret_cast<const double2*>(sigma),
        reinterpret_cast<const double2*>(u), n, reinterpret_cast<double2*>(lam));
}

}  // namespace magb
