// kernels_nersc.cu -- device side of NERSC configuration I/O
// (export_config_nersc / import_config_nersc, field-matrix.h:452-713).
//
// The payload of a NERSC file is the lattice in lexicographic site order
// (x0 fastest), four links per site, each link its first two rows
// (DATATYPE 4D_SU3_GAUGE, 6 complex) or all three (4D_SU3_GAUGE_3x3,
// 9 complex), every real an IEEE-754 binary64 in big-endian byte order.
// The whole payload is staged in device memory and these kernels work on it
// in place: byte order, the 32-bit word checksum, segment CRC-32 values, and
// the conversion to and from the link tiles.  All are bound by HBM bandwidth.
#include <stdint.h>

#include "kernels.h"

namespace magb {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ uint64_t bswap64(uint64_t w) {
    const uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32);
    return ((uint64_t)__byte_perm(lo, 0, 0x0123) << 32) | (uint64_t)__byte_perm(hi, 0, 0x0123);
}

__device__ __forceinline__ uint32_t words32(uint64_t w) { return (uint32_t)w + (uint32_t)(w >> 32); }

// sum of 32-bit words modulo 2^32 over the block, added to *sum (exact: the
// sum is associative and commutative modulo 2^32, so the result is
// independent of the launch shape)
__device__ __forceinline__ void add_block_sum(uint32_t v, unsigned int* sum) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __shared__ uint32_t sm[kBlock / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) atomicAdd(sum, v);
    }
}

// n16 = payload bytes / 16.  to_host = 1: big-endian file words -> host order,
// checksum of the host-order words; to_host = 0: checksum of the host-order
// words, then -> big-endian.
__global__ void k_swap64_sum32(ulonglong2* p, size_t n16, int to_host, unsigned int* sum) {
    uint32_t s = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += stride) {
        ulonglong2 v = p[i];
        if (to_host) {
            v.x = bswap64(v.x);
            v.y = bswap64(v.y);
            s += words32(v.x) + words32(v.y);
        } else {
            s += words32(v.x) + words32(v.y);
            v.x = bswap64(v.x);
            v.y = bswap64(v.y);
        }
        p[i] = v;
    }
    add_block_sum(s, sum);
}

// CRC-32 of the IEEE 802.3 / zlib polynomial (reflected 0xEDB88320), register
// started at 0 and not complemented, of each `seg`-byte segment (the last one
// may be shorter); the host chains the segment values with the linear
// zero-byte shift.  Slicing by four: tab[k][b] is the register after byte b
// followed by k zero bytes.
__global__ void k_crc32_segments(const uint8_t* p, size_t n, size_t seg, uint32_t* z, size_t nseg) {
    __shared__ uint32_t tab[4][256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) {
        uint32_t c = (uint32_t)b;
        for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
        tab[0][b] = c;
    }
    __syncthreads();
    for (int k = 1; k < 4; k++) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) {
            const uint32_t c = tab[k - 1][b];
            tab[k][b] = (c >> 8) ^ tab[0][c & 0xffu];
        }
        __syncthreads();
    }
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseg) return;
    const size_t b0 = i * seg;
    const size_t b1 = b0 + seg < n ? b0 + seg : n;
    uint32_t c = 0;
    size_t b = b0;
    // segments start on multiples of 16 bytes (seg is a multiple of 16); four
    // independent 16-byte loads are in flight before the table steps
    const uint4* q = reinterpret_cast<const uint4*>(p + b0);
    for (; b + 64 <= b1; b += 64, q += 4) {
        uint4 v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) v[j] = q[j];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t w[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                c ^= w[k];
                c = tab[3][c & 0xffu] ^ tab[2][(c >> 8) & 0xffu] ^ tab[1][(c >> 16) & 0xffu] ^ tab[0][c >> 24];
            }
        }
    }
    for (; b + 16 <= b1; b += 16, q++) {
        const uint4 v = *q;
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            c ^= w[k];
            c = tab[3][c & 0xffu] ^ tab[2][(c >> 8) & 0xffu] ^ tab[1][(c >> 16) & 0xffu] ^ tab[0][c >> 24];
        }
    }
    for (; b < b1; b++) c = (c >> 8) ^ tab[0][(c ^ p[b]) & 0xffu];
    z[i] = c;
}

// z2[g] = fold of the registers z[g*G .. min((g+1)*G, n)) of consecutive
// equal-length segments: r <- S(r) ^ z[j] from r = 0, S the register advance
// over one segment of zero bytes given as four byte tables (tab[k][b])
__global__ void k_crc32_fold(const uint32_t* z, size_t n, int G, const uint32_t* tab, uint32_t* z2, size_t ngroups) {
    __shared__ uint32_t t[4][256];
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) t[i >> 8][i & 255] = tab[i];
    __syncthreads();
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    const size_t j0 = g * (size_t)G;
    const size_t j1 = j0 + G < n ? j0 + G : n;
    uint32_t r = 0;
    for (size_t j = j0; j < j1; j++)
        r = t[0][r & 0xffu] ^ t[1][(r >> 8) & 0xffu] ^ t[2][(r >> 16) & 0xffu] ^ t[3][r >> 24] ^ z[j];
    z2[g] = r;
}

// Payload <-> link tiles through shared memory: a block owns 32 consecutive
// sites (one link tile per direction); the payload of those sites is one
// contiguous run of 32 * 4 * NC * 16 bytes, moved with coalesced 16-byte
// accesses, while the tiles are read or written one coalesced element plane
// at a time.  In shared memory each site's 4 * NC values are followed by one
// pad slot, so the 32 sites of a warp start on distinct bank groups.
constexpr int kTileSites = 32;
constexpr int kConvThreads = 128;

template <int NC>
__device__ __forceinline__ int smem_slot(int i) {  // payload value i of the block -> shared slot
    return i + i / (4 * NC);
}

// payload (host order) -> link tiles of one chain; NC = 6 rebuilds the third
// row with the reference's reunitarize (field-matrix.h:83-100: CPS Unitarize
// of rows 0, 1 unless both are zero), as import_config_nersc does after
// copying the truncated matrices (field-matrix.h:680-690)
template <int NC>
__global__ void __launch_bounds__(kConvThreads) k_payload_to_links(const double* pay, int off, int V,
                                                                   LinkPlanes<double> U) {
    __shared__ double2 sm[kTileSites * (4 * NC + 1)];
    const int s0 = blockIdx.x * kTileSites;
    const int ns = min(kTileSites, V - s0);
    const double2* src = reinterpret_cast<const double2*>(pay) + (size_t)s0 * 4 * NC;
    for (int i = threadIdx.x; i < ns * 4 * NC; i += kConvThreads) sm[smem_slot<NC>(i)] = src[i];
    __syncthreads();
    // thread = (mu, site) with the site fastest: the stores of one element are one coalesced plane
    const int mu = threadIdx.x / kTileSites, ls = threadIdx.x % kTileSites;
    if (ls >= ns) return;
    const double2* a = sm + ls * (4 * NC + 1) + mu * NC;
    mat3<double> m;
    set_zero(m);
#pragma unroll
    for (int k = 0; k < NC; k++) m.e[k / 3][k % 3] = mk(a[k].x, a[k].y);
    if (NC == 6) {
        bool all_zero = true;
#pragma unroll
        for (int k = 0; k < 6; k++) all_zero = all_zero && m.e[k / 3][k % 3].re == 0.0 && m.e[k / 3][k % 3].im == 0.0;
        if (!all_zero) unitarize(m);
    }
    U.store(mu, off + s0 + ls, m);
}

template <int NC>
__global__ void __launch_bounds__(kConvThreads) k_links_to_payload(LinkPlanes<double> U, int off, int V,
                                                                   double* pay) {
    __shared__ double2 sm[kTileSites * (4 * NC + 1)];
    const int s0 = blockIdx.x * kTileSites;
    const int ns = min(kTileSites, V - s0);
    const int mu = threadIdx.x / kTileSites, ls = threadIdx.x % kTileSites;
    if (ls < ns) {
        const mat3<double> m = U.load(mu, off + s0 + ls);
        double2* a = sm + ls * (4 * NC + 1) + mu * NC;
#pragma unroll
        for (int k = 0; k < NC; k++) a[k] = make_double2(m.e[k / 3][k % 3].re, m.e[k / 3][k % 3].im);
    }
    __syncthreads();
    double2* dst = reinterpret_cast<double2*>(pay) + (size_t)s0 * 4 * NC;
    for (int i = threadIdx.x; i < ns * 4 * NC; i += kConvThreads) dst[i] = sm[smem_slot<NC>(i)];
}

unsigned grid_for(size_t n, unsigned cap) {
    const size_t b = (n + kBlock - 1) / kBlock;
    return (unsigned)(b < cap ? (b ? b : 1) : cap);
}

}  // namespace

void launch_swap64_sum32(void* payload, size_t bytes, bool to_host, unsigned int* sum, cudaStream_t s) {
    const size_t n16 = bytes / 16;
    // 148 SMs x 8 resident blocks of 256 threads: a grid-stride loop over the payload
    k_swap64_sum32<<<grid_for(n16, 148 * 8), kBlock, 0, s>>>(static_cast<ulonglong2*>(payload), n16,
                                                              to_host ? 1 : 0, sum);
}

void launch_crc32_segments(const void* payload, size_t bytes, size_t seg, uint32_t* z, cudaStream_t s) {
    const size_t nseg = (bytes + seg - 1) / seg;
    k_crc32_segments<<<grid_for(nseg, 1u << 30), kBlock, 0, s>>>(static_cast<const uint8_t*>(payload), bytes, seg,
                                                                 z, nseg);
}

void launch_crc32_fold(const uint32_t* z, size_t n, int G, const uint32_t* tab, uint32_t* z2, cudaStream_t s) {
    const size_t ng = (n + G - 1) / G;
    if (ng == 0) return;
    k_crc32_fold<<<grid_for(ng, 1u << 30), kBlock, 0, s>>>(z, n, G, tab, z2, ng);
}

void launch_payload_to_links(const double* payload, int two_row, int off, int V, LinkPlanes<double> U,
                             cudaStream_t s) {
    const unsigned grid = (unsigned)((V + kTileSites - 1) / kTileSites);
    if (two_row) k_payload_to_links<6><<<grid, kConvThreads, 0, s>>>(payload, off, V, U);
    else k_payload_to_links<9><<<grid, kConvThreads, 0, s>>>(payload, off, V, U);
}

void launch_links_to_payload(LinkPlanes<double> U, int two_row, int off, int V, double* payload, cudaStream_t s) {
    const unsigned grid = (unsigned)((V + kTileSites - 1) / kTileSites);
    if (two_row) k_links_to_payload<6><<<grid, kConvThreads, 0, s>>>(U, off, V, payload);
    else k_links_to_payload<9><<<grid, kConvThreads, 0, s>>>(U, off, V, payload);
}

}  // namespace magb
