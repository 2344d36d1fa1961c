// kernels_wloop.cu -- Wilson loops (field-wloop.h:26-99) and the constrained
// plaquette (field-matrix.h:407-443), FP64 with double-double sums.
//
// Planar R x T loops reuse line products: for one spatial direction i the
// lines S_R(x) = U_i(x) ... U_i(x+(R-1)i) are built once for R = 1..Rmax; the
// temporal line T_T(x) grows by one link per T; then
//   W_i(R,T)(x) = ReTr( S_R(x) T_T(x+R i) S_R(x+T t)^dag T_T(x)^dag )
// costs two products and one trace per (x, R, T) instead of 2(R+T)-1 products.
#include "gauge_ops.cuh"
#include "kernels.h"

namespace magb {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ bool locate(const DevGeom& g, int gs, ChainInfo& ci, Site& st) {
    if (gs >= g.vpad) return false;
    ci = g.chains[g.c2c[gs / MAG_CHUNK]];
    const int s = gs - ci.off;
    if (s >= ci.V) return false;
    decode(ci, s, st);
    return true;
}

__device__ __forceinline__ int wrap_shift(const ChainInfo& ci, int xd, int d, int k) {
    int w = (xd + k) % ci.L[d];
    if (w < 0) w += ci.L[d];
    return (w - xd) * ci.stride[d];
}

__device__ __forceinline__ dd2 two_sum(double a, double b) {
    const double s = a + b, bp = s - a;
    return dd2{s, (a - (s - bp)) + (b - bp)};
}
__device__ __forceinline__ dd2 dd_add(dd2 a, dd2 b) {
    dd2 s = two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return two_sum(s.hi, s.lo);
}
__device__ dd2 block_reduce(dd2 v) {
    __shared__ dd2 sm[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dd2 w{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
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
            dd2 w{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
            v = dd_add(v, w);
        }
    }
    return v;
}

// line(x) <- prev(x) U_d(x + k d)   (prev = nullptr: line(x) = U_d(x))
__global__ void k_line_extend(DevGeom g, LinkPlanes<double> U, int d, LinkPlanes<double> prev, int k,
                              LinkPlanes<double> out) {
    ChainInfo ci;
    Site st;
    if (!locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st)) return;
    const mat3<double> u = U.load(d, st.g + wrap_shift(ci, st.x[d], d, k));
    out.store(0, st.g, prev.p ? mul(prev.load(0, st.g), u) : u);
}

// partial[block * Rmax + R-1] = sum_x ReTr W_i(R, T)(x).  The R values are
// taken four at a time: a thread forms its site's four loops (their loads
// issued together) and the block reduces the four sums at once, instead of one
// block reduction (two barriers) per R.  ReTr(S_R(x) T(x+Ri) S_R(x+Tt)^dag
// T(x)^dag) = ReTr(a c^dag) with a = S_R(x) T(x+Ri), c = T(x) S_R(x+Tt): two
// products and one trace of a product per loop.
constexpr int kRChunk = 4;
__global__ void __launch_bounds__(kBlock, 2) k_wloop_accum(DevGeom g, LinkPlanes<double> lines, int Rmax,
                                                           LinkPlanes<double> tl, int i, int T, dd2* partial) {
    __shared__ dd2 sm[kBlock / 32][kRChunk];
    ChainInfo ci;
    Site st;
    const bool ok = locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st);
    int gT = 0, gR = 0;
    if (ok) {
        gT = st.g + wrap_shift(ci, st.x[3], 3, T);
        gR = st.x[i];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int R0 = 1; R0 <= Rmax; R0 += kRChunk) {
        double v[kRChunk];
#pragma unroll
        for (int r = 0; r < kRChunk; r++) {
            const int R = R0 + r;
            v[r] = 0.0;
            if (ok && R <= Rmax) {
                const LinkPlanes<double> S{lines.p + (size_t)(R - 1) * 9 * lines.vpad, lines.vpad};
                const mat3<double> a = mul(S.load(0, st.g), tl.load(0, st.g + wrap_shift(ci, gR, i, R)));
                const mat3<double> c = mul(tl.load(0, st.g), S.load(0, gT));
                v[r] = retr_mul_nd(a, c);
            }
        }
#pragma unroll
        for (int r = 0; r < kRChunk; r++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[r] += __shfl_down_sync(0xffffffffu, v[r], o);
        __syncthreads();  // the previous chunk's sums have been read
        if (lane == 0)
#pragma unroll
            for (int r = 0; r < kRChunk; r++) sm[wid][r] = dd2{v[r], 0.0};
        __syncthreads();
        if (threadIdx.x < kRChunk && R0 + (int)threadIdx.x <= Rmax) {
            dd2 s = sm[0][threadIdx.x];
            for (int w = 1; w < kBlock / 32; w++) s = dd_add(s, sm[w][threadIdx.x]);
            partial[(size_t)blockIdx.x * Rmax + R0 - 1 + threadIdx.x] = s;
        }
    }
}

// generic closed paths from every site (or from coarse sites when mag > 0):
// sum over paths of ReTr of the path-ordered product (get_path_ordered_product,
// field-matrix.h:102-131); dirs: 0..3 forward, 4..7 backward
__global__ void k_paths(DevGeom g, LinkPlanes<double> U, const int* dirs, int npath, int plen, int coarse_mag,
                        dd2* partial) {
    ChainInfo ci;
    Site st;
    dd2 v{0.0, 0.0};
    if (locate(g, blockIdx.x * blockDim.x + threadIdx.x, ci, st)) {
        bool active = true;
        if (coarse_mag > 0)
            for (int d = 0; d < 4; d++) active = active && (st.x[d] % coarse_mag == 0);
        if (active) {
            double acc = 0.0;
            for (int p = 0; p < npath; p++) {
                int y[4] = {st.x[0], st.x[1], st.x[2], st.x[3]};
                int gy = st.g;
                mat3<double> m = unit_mat<double>();
                for (int k = 0; k < plen; k++) {
                    const int d = dirs[p * plen + k];
                    if (d < 0) break;
                    if (d < 4) {
                        m = mul(m, U.load(d, gy));
                        const int sh = wrap_shift(ci, y[d], d, 1);
                        gy += sh;
                        y[d] = y[d] + 1 < ci.L[d] ? y[d] + 1 : 0;
                    } else {
                        const int e = d - 4;
                        const int sh = wrap_shift(ci, y[e], e, -1);
                        gy += sh;
                        y[e] = y[e] > 0 ? y[e] - 1 : ci.L[e] - 1;
                        m = mul_nd(m, U.load(e, gy));
                    }
                }
                acc += retr(m);
            }
            v.hi = acc;
        }
    }
    v = block_reduce(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

// per chain: out[c * nq + q] = sum of partial[b * nq + q] over the chain's blocks
__global__ void k_finalize_multi(DevGeom g, const dd2* partial, int nq, dd2* out) {
    const int c = blockIdx.x;
    const ChainInfo ci = g.chains[c];
    const int b0 = ci.off / kBlock, b1 = (ci.off + ci.V + kBlock - 1) / kBlock;
    for (int q = 0; q < nq; q++) {
        dd2 v{0.0, 0.0};
        for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) v = dd_add(v, partial[(size_t)b * nq + q]);
        v = block_reduce(v);
        if (threadIdx.x == 0) out[c * nq + q] = v;
        __syncthreads();
    }
}

unsigned blocks(const DevGeom& g) { return (unsigned)((g.vpad + kBlock - 1) / kBlock); }

}  // namespace

// lines: Rmax consecutive single-direction planes (9 * vpad complex each);
// tl, tl2: two single-direction planes for the temporal line (ping-pong).
// out[((i * Tmax + T-1) * nchain + c) * Rmax + R-1] = sum over the chain's sites
// of ReTr W_i(R, T) for spatial direction i; partial holds blocks * Rmax entries.
void launch_wilson_planar(const DevGeom& g, LinkPlanes<double> U, int Rmax, int Tmax, LinkPlanes<double> lines,
                          LinkPlanes<double> tl, LinkPlanes<double> tl2, dd2* partial, dd2* out, cudaStream_t s) {
    const unsigned nb = blocks(g);
    for (int i = 0; i < 3; i++) {
        for (int R = 1; R <= Rmax; R++) {
            LinkPlanes<double> cur{lines.p + (size_t)(R - 1) * 9 * lines.vpad, lines.vpad};
            LinkPlanes<double> prev{R > 1 ? lines.p + (size_t)(R - 2) * 9 * lines.vpad : nullptr, lines.vpad};
            k_line_extend<<<nb, kBlock, 0, s>>>(g, U, i, prev, R - 1, cur);
        }
        LinkPlanes<double> a = tl, b = tl2;
        for (int T = 1; T <= Tmax; T++) {
            k_line_extend<<<nb, kBlock, 0, s>>>(g, U, 3, T > 1 ? a : LinkPlanes<double>{nullptr, 0}, T - 1, b);
            k_wloop_accum<<<nb, kBlock, 0, s>>>(g, lines, Rmax, b, i, T, partial);
            k_finalize_multi<<<g.nchain, kBlock, 0, s>>>(g, partial, Rmax,
                                                         out + (size_t)(i * Tmax + (T - 1)) * g.nchain * Rmax);
            LinkPlanes<double> t = a;
            a = b;
            b = t;
        }
    }
}

void launch_wilson_general(const DevGeom& g, LinkPlanes<double> U, const int* dirs, int npath, int plen,
                           int coarse_mag, dd2* partial, dd2* out, cudaStream_t s) {
    k_paths<<<blocks(g), kBlock, 0, s>>>(g, U, dirs, npath, plen, coarse_mag, partial);
    k_finalize_multi<<<g.nchain, kBlock, 0, s>>>(g, partial, 1, out);
}

}  // namespace magb
