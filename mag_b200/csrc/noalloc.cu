// noalloc.cu -- gauge-action sums without any device allocation.
//
// Who needs this: code that cannot call cudaMalloc itself, for example a
// lattice driver that hands this library a slice of a device pool it manages
// (every byte accounted for up front), or a latency-sensitive loop that must
// not pay for cudaMalloc's implicit device synchronisation.  Such a caller
// already holds the links in device memory and only wants the plaquette and
// rectangle sums of total_plaq / total_rectangular (field-matrix.h:299-385).
//
// The per-block partial sums live in a fixed file-scope device array sized
// for MAG_NOALLOC_MAX_SITES sites (2 MiB).  Every GPU that loads the library
// holds that array until the process exits, and every call on a device shares
// it: two calls that overlap on the GPU (different streams, no ordering
// between them) race on it and both results are then undefined.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/mag_c.h"
#include "gauge_ops.cuh"
#include "kernels.h"

using namespace magb;

namespace magb {
void set_last_error(const std::string& msg);  // mag_api.cu
}

namespace {

constexpr int kBlock = 256;
constexpr int kMaxBlocks = MAG_NOALLOC_MAX_SITES / kBlock;

// two double-double partials (plaquette, rectangle) per block
__device__ __align__(256) dd2 g_noalloc_partials[2 * kMaxBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
dd2* g_partials_ptr[kMaxDevices] = {};
CUcontext g_partials_ctx[kMaxDevices] = {};  // the context each cached address belongs to

__device__ __forceinline__ dd2 na_two_sum(double a, double b) {
    const double s = a + b, bp = s - a;
    return dd2{s, (a - (s - bp)) + (b - bp)};
}
__device__ __forceinline__ dd2 na_add(dd2 a, dd2 b) {
    dd2 s = na_two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return na_two_sum(s.hi, s.lo);
}
__device__ dd2 na_block_reduce(dd2 v) {
    __shared__ dd2 sm[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dd2 w{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
        v = na_add(v, w);
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
            v = na_add(v, w);
        }
    }
    return v;
}

// links in the reference's AoS layout double[V][4][3][3][2]
__device__ __forceinline__ mat3<double> aos_link(const double* a, int s, int mu) {
    const double* q = a + ((long)s * 4 + mu) * 18;
    mat3<double> m;
#pragma unroll
    for (int k = 0; k < 9; k++) m.e[k / 3][k % 3] = mk(q[2 * k], q[2 * k + 1]);
    return m;
}

// ReTr of the six plaquettes and twelve rectangles at one site
// (get_plaq, field-matrix.h:202-221; get_rectangular, field-matrix.h:249-297)
__global__ void k_noalloc_partials(ChainInfo ci, const double* links, dd2* partials) {
    dd2 p{0.0, 0.0}, r{0.0, 0.0};
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < ci.V) {
        Site st;
        decode(ci, s, st);
        double ps = 0.0, rs = 0.0;
        for (int mu = 1; mu < 4; mu++) {
            const mat3<double> umu = aos_link(links, s, mu);
            const int gm = nb(ci, st, mu, 1);
            for (int nu = 0; nu < mu; nu++) {
                const mat3<double> unu = aos_link(links, s, nu);
                const int gn = nb(ci, st, nu, 1);
                const int gmn = nb(ci, st, mu, 1, nu, 1);
                const mat3<double> m = mul(umu, aos_link(links, gm, nu));
                const mat3<double> n = mul(unu, aos_link(links, gn, mu));
                ps += retr(mul_nd(m, n));
                mat3<double> a = mul(mul(umu, aos_link(links, gm, nu)), aos_link(links, gmn, nu));
                mat3<double> b = mul(mul(unu, aos_link(links, gn, nu)), aos_link(links, nb(ci, st, nu, 2), mu));
                rs += retr(mul_nd(b, a));
                a = mul(mul(umu, aos_link(links, gm, mu)), aos_link(links, nb(ci, st, mu, 2), nu));
                b = mul(mul(unu, aos_link(links, gn, mu)), aos_link(links, gmn, mu));
                rs += retr(mul_nd(b, a));
            }
        }
        p.hi = ps;
        r.hi = rs;
    }
    p = na_block_reduce(p);
    r = na_block_reduce(r);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = p;
        partials[2 * blockIdx.x + 1] = r;
    }
}

// one block: sum the partials of every block in block order
__global__ void k_noalloc_finalize(int nblocks, const dd2* partials, double* out) {
    for (int q = 0; q < 2; q++) {
        dd2 v{0.0, 0.0};
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = na_add(v, partials[2 * b + q]);
        v = na_block_reduce(v);
        if (threadIdx.x == 0) out[q] = v.hi + v.lo;
        __syncthreads();
    }
}

int na_fail(int code, const std::string& msg) {
    set_last_error(msg);  // reported by mag_last_error()
    return code;
}

// The calling thread's current CUDA context, through the driver entry point
// the runtime hands out (no link-time dependence on the driver library).
typedef CUresult (*ctx_get_current_fn)(CUcontext*);
CUcontext current_context() {
    static ctx_get_current_fn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        fn = reinterpret_cast<ctx_get_current_fn>(p);
    }
    CUcontext c = nullptr;
    return fn(&c) == CUDA_SUCCESS ? c : nullptr;
}

// Device address of the static partials for the current device.  The first
// call on a device (in a given context) looks it up with cudaGetSymbolAddress;
// later calls in the same context reuse it.  A call made under another
// context on the same device looks the address up again for that context.
int partials_for_current_device(dd2** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(MAG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return na_fail(MAG_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_ptr[dev] || g_partials_ctx[dev] != current_context()) {
        void* p = nullptr;
        // also makes the device's primary context current if no context was
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            return na_fail(MAG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_partials_ptr[dev] = static_cast<dd2*>(p);
        g_partials_ctx[dev] = current_context();
    }
    *out = g_partials_ptr[dev];
    return MAG_OK;
}

}  // namespace

extern "C" int mag_action_sums_noalloc(const int dims[4], const double* d_links, double* d_sums, void* stream) {
    if (!dims || !d_links || !d_sums) return na_fail(MAG_ERR_ARG, "mag_action_sums_noalloc: null argument");
    ChainInfo ci{};
    long V = 1;
    for (int d = 0; d < 4; d++) {
        if (dims[d] < 2) return na_fail(MAG_ERR_ARG, "mag_action_sums_noalloc: every extent must be >= 2");
        ci.L[d] = dims[d];
        ci.stride[d] = (int)V;
        V *= dims[d];
        if (V > MAG_NOALLOC_MAX_SITES)
            return na_fail(MAG_ERR_ARG, "mag_action_sums_noalloc: lattice exceeds the " +
                                            std::to_string(MAG_NOALLOC_MAX_SITES) +
                                            "-site limit of its static scratch; use mag_action");
    }
    set_divisors(ci);
    ci.V = (int)V;
    ci.L3g = ci.hi3 = ci.L[3];
    ci.Vg = (int)V;
    dd2* partials = nullptr;
    const int r = partials_for_current_device(&partials);
    if (r != MAG_OK) return r;
    const int nblocks = (int)((V + kBlock - 1) / kBlock);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_noalloc_partials<<<nblocks, kBlock, 0, s>>>(ci, d_links, partials);
    k_noalloc_finalize<<<1, kBlock, 0, s>>>(nblocks, partials, d_sums);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(MAG_ERR_CUDA, std::string("mag_action_sums_noalloc: ") + cudaGetErrorString(e));
    return MAG_OK;
}
