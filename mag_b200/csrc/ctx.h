// ctx.h -- the context behind the C ABI of libmag_b200.so (internal to the library).
//
// mag_ctx owns every device buffer and one stream.  The integrator is the
// force-gradient scheme of field-hmc.h:525-567 (or the leapfrog of :569-587)
// written as a fixed launch sequence with device-resident scalars, so one HMC
// trajectory (momenta, H_old, integration, reunitarisation, H_new, accept,
// restore, record) replays as a single CUDA graph with no host round trip.
// The C ABI over it is split by subsystem: mag_api.cu (contexts, forces, MD,
// trajectories, measurements, the tuner), mag_nersc_api.cu (configuration
// files), mag_dd.cu (a lattice split into slabs along x3) and mag_multi_api.cu
// (the two-level coupling).
#pragma once
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <functional>
#include <cstring>
#include <string>
#include <thread>
#include <condition_variable>
#include <mutex>
#include <memory>
#include <vector>

#include "../../include/mag_c.h"
#include "../../include/mag_diag.h"
#include "kernels.h"
#include "nersc_host.h"

using namespace magb;

namespace magb {

// sets the message mag_last_error() returns (mag_api.cu)
void set_last_error(const std::string& msg);

// records msg for mag_last_error() and returns code
inline int fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

#define MAG_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(MAG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

#define MAG_TRY(call)              \
    do {                           \
        int r_ = (call);           \
        if (r_ != MAG_OK) return r_; \
    } while (0)

constexpr int kHistCap = 256;

template <typename T>
struct StoutBufs {
    std::vector<LinkPlanes<T>> lv;   // lv[k] = links after k+1 stout levels
    std::vector<AlgPlanes<T>> Q;     // Q[k] = exponent of level k -> k+1
    AlgPlanes<T> lam{nullptr, 0};
    LinkPlanes<T> za{nullptr, 0}, zp{nullptr, 0};
};

// host double-double helpers (final action values)
struct hdd {
    double hi, lo;
};
inline hdd h_two_sum(double a, double b) {
    const double s = a + b, bp = s - a;
    return hdd{s, (a - (s - bp)) + (b - bp)};
}
inline hdd h_add(hdd a, hdd b) {
    hdd s = h_two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return h_two_sum(s.hi, s.lo);
}
inline hdd h_mul(hdd a, double b) {
    const double p = a.hi * b;
    const double e = std::fma(a.hi, b, -p);
    return h_two_sum(p, e + a.lo * b);
}
inline hdd h_neg(hdd a) { return hdd{-a.hi, -a.lo}; }

// CRC segments of a configuration file: about two per resident thread of a 148-SM
// device, at least 256 bytes each (mag_nersc_api.cu)
constexpr size_t kCrcThreads = 148 * 2048 * 2;
constexpr int kCrcGroup = 64;  // segment registers folded per thread on the device
inline size_t crc_seg(size_t bytes) {
    const size_t s = (bytes + kCrcThreads - 1) / kCrcThreads;
    return std::max<size_t>(256, (s + 15) / 16 * 16);
}
}  // namespace magb

struct mag_ctx;
namespace magb {
int nersc_buffers(mag_ctx* ctx);            // pinned staging and CRC buffers (mag_nersc_api.cu)
int ensure_crc_tab(mag_ctx* ctx, size_t seg);
}  // namespace magb

// Halo exchange of a lattice decomposed along x3 (see mag_dd_create): called at
// every point where a kernel is about to read neighbour links, momenta-derived
// fields or Lambda across a shard boundary, and where the Hamiltonian's sums
// must become whole-lattice sums.  Undivided contexts have no hook.
struct HaloHook {
    virtual ~HaloHook() {}
    // fill the halo slabs of a field of 4 planes, `unit` bytes per site per plane
    virtual int exchange(mag_ctx* c, void* base, size_t unit) = 0;
    // sum the listed slots of the context's sums over all shards (and the
    // reunitarisation deviation's maximum when `reunit`)
    virtual int reduce(mag_ctx* c, const int* slots, int nslots, bool reunit) = 0;
};

struct mag_ctx {
    mag_params p{};
    std::vector<mag_params> cp;
    std::vector<ChainInfo> hc;
    int nchain = 0;
    long vpad = 0;
    bool iwasaki = true, mixed = false, any_mag = false;
    cudaStream_t stream = nullptr;
    DevGeom geom{};
    std::vector<void*> allocs;
    size_t bytes = 0;

    ChainInfo* d_chains = nullptr;
    uint16_t* d_c2c = nullptr;
    unsigned long long* d_stream_index = nullptr;
    LinkPlanes<double> U{nullptr, 0}, Ubak{nullptr, 0}, Uaux{nullptr, 0};
    AlgPlanes<double> P{nullptr, 0}, F{nullptr, 0};
    LinkPlanes<float> U32{nullptr, 0}, Uaux32{nullptr, 0};
    AlgPlanes<float> F32{nullptr, 0};
    StoutBufs<double> st64;
    StoutBufs<float> st32;
    dd2* partial = nullptr;
    dd2* sums = nullptr;
    ChainState* cstate = nullptr;
    unsigned long long* reunit = nullptr;
    TrajRecord* rec = nullptr;
    TrajRecord* hist = nullptr;
    long long* hist_base = nullptr;
    long long* traj_counter = nullptr;
    long long* tmp_counter = nullptr;
    double* d_uniform = nullptr;
    bool uniform_override = false;
    double* staging = nullptr;
    long max_v = 0;
    // NERSC I/O: pinned double buffer, CRC segment registers, word checksum
    nersc::Pinned pin;
    DemonTables* d_demon_tables = nullptr;  // per-link demon sweep: staple paths through the site window
    DemonState* d_demon = nullptr;          // one per chain
    DemonJob* d_demon_jobs = nullptr;       // one per chain
    double* demon_aos = nullptr;            // AoS copy of every chain (sweeps of the whole ensemble)
    std::vector<unsigned long long> h_stream_index;
    uint32_t* d_crc = nullptr;      // segment registers (kCrcThreads + 1)
    uint32_t* d_crc2 = nullptr;     // folded groups
    uint32_t* d_crc_tab = nullptr;  // 4 x 256 shift tables of one segment
    size_t crc_tab_seg = 0;         // segment length the tables hold
    unsigned int* d_csum = nullptr;
    long long host_traj = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_run_ms = 0.0;
    double last_measure_ms = 0.0;

    // domain decomposition along x3: shard `shard_rank` of `shard_n`, halo depth `shard_h` (0: undivided)
    HaloHook* halo = nullptr;
    int shard_n = 1, shard_rank = 0, shard_h = 0;
    int halo_rc = MAG_OK;
    // The hook is called at every exchange point even after a failure (the first
    // status is kept): the other shards meet this one there.
    template <typename T>
    void hx(LinkPlanes<T> l) {
        if (!halo) return;
        const int r = halo->exchange(this, l.p, sizeof(cplx<T>) * LinkPlanes<T>::kElems);
        if (halo_rc == MAG_OK) halo_rc = r;
    }
    template <typename T>
    void hx(AlgPlanes<T> a) {
        if (!halo) return;
        const int r = halo->exchange(this, a.p, sizeof(T) * 8);
        if (halo_rc == MAG_OK) halo_rc = r;
    }
    void hreduce(std::initializer_list<int> slots, bool reunit_max) {
        if (!halo) return;
        std::vector<int> v(slots);
        const int r = halo->reduce(this, v.data(), (int)v.size(), reunit_max);
        if (halo_rc == MAG_OK) halo_rc = r;
    }

    ~mag_ctx() {
        delete halo;
        halo = nullptr;
        release();
    }

    void release() {
        pin.release();
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (void* a : allocs) cudaFree(a);
        allocs.clear();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        ev0 = ev1 = nullptr;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    int alloc(void** ptr, size_t n) {
        cudaError_t e = cudaMalloc(ptr, n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(MAG_ERR_NOMEM, "cudaMalloc(" + std::to_string(n) + " bytes): " + cudaGetErrorString(e));
        }
        allocs.push_back(*ptr);
        bytes += n;
        return MAG_OK;
    }
    template <typename T>
    int alloc_links(LinkPlanes<T>& l) {
        l.vpad = vpad;
        return alloc((void**)&l.p, sizeof(cplx<T>) * 4 * LinkPlanes<T>::kElems * (size_t)vpad);
    }
    template <typename T>
    int alloc_alg(AlgPlanes<T>& a) {
        a.vpad = vpad;
        return alloc((void**)&a.p, sizeof(T) * 32 * (size_t)vpad);
    }
    template <typename T>
    int alloc_stout(StoutBufs<T>& b, bool backward) {
        b.lv.resize(p.n_stout);
        b.Q.resize(p.n_stout);
        for (int k = 0; k < p.n_stout; k++) {
            MAG_TRY(alloc_links(b.lv[k]));
            MAG_TRY(alloc_alg(b.Q[k]));
        }
        if (backward && p.n_stout > 0) {
            MAG_TRY(alloc_alg(b.lam));
            MAG_TRY(alloc_links(b.za));
            MAG_TRY(alloc_links(b.zp));
        }
        return MAG_OK;
    }

    int check(const char* what) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(MAG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        return MAG_OK;
    }
    int sync(const char* what) {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return fail(MAG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        return check(what);
    }

    // shard != nullptr: {nshards, rank, halo} of a lattice split along x3 (n == 1)
    int init(const mag_params* params, int n, const int* shard = nullptr) {
        p = params[0];
        nchain = n;
        if (shard) {
            shard_n = shard[0];
            shard_rank = shard[1];
            shard_h = shard[2];
        }
        iwasaki = p.action == MAG_ACTION_IWASAKI;
        mixed = p.precision == MAG_PREC_MIXED;
        long off = 0;
        for (int c = 0; c < n; c++) {
            const mag_params& q = params[c];
            ChainInfo ci{};
            long V = 1;
            for (int d = 0; d < 4; d++) {
                if (q.dims[d] < 2) return fail(MAG_ERR_ARG, "every lattice extent must be >= 2");
                if (q.mag < 0 || (q.mag > 0 && q.dims[d] % q.mag != 0))
                    return fail(MAG_ERR_ARG, "lattice extents must be divisible by mag");
                ci.L[d] = q.dims[d];
                ci.stride[d] = (int)V;
                V *= q.dims[d];
            }
            if (q.mag == 1) return fail(MAG_ERR_ARG, "mag = 1 freezes every link (field-hmc.h:331); use 0 or >= 2");
            if (q.action != p.action) return fail(MAG_ERR_ARG, "all chains of an ensemble share the action type");
            set_divisors(ci);
            ci.V = (int)V;
            ci.off = (int)off;
            ci.mag = q.mag;
            ci.org3 = 0;
            ci.L3g = ci.L[3];
            ci.lo3 = 0;
            ci.hi3 = ci.L[3];
            ci.Vg = (int)V;
            if (shard_h > 0) {
                // the shard holds lattice x3 in [rank Lloc - h, (rank + 1) Lloc + h): interior and halos
                const int L3 = q.dims[3], loc = L3 / shard_n;
                ci.L[3] = loc + 2 * shard_h;
                V = (long)ci.L[0] * ci.L[1] * ci.L[2] * ci.L[3];
                ci.V = (int)V;
                ci.org3 = shard_rank * loc - shard_h;
                ci.L3g = L3;
                ci.lo3 = shard_h;
                ci.hi3 = shard_h + loc;
                ci.Vg = ci.L[0] * ci.L[1] * ci.L[2] * L3;
            }
            ci.beta = q.beta;
            ci.c1 = iwasaki ? q.c1 : 0.0;
            ci.c0 = 1.0 - 8.0 * ci.c1;
            ci.rho = q.rho;
            hc.push_back(ci);
            cp.push_back(q);
            any_mag = any_mag || q.mag > 0;
            max_v = std::max(max_v, V);
            off += (V + MAG_CHUNK - 1) / MAG_CHUNK * MAG_CHUNK;
        }
        if (off >= (1L << 31) / 36) return fail(MAG_ERR_ARG, "total volume too large for 32-bit site indices");
        if (p.n_steps < 1 || p.n_stout < 0 || p.n_stout > 8) return fail(MAG_ERR_ARG, "bad n_steps or n_stout");
        vpad = off;
        MAG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        MAG_CUDA(cudaEventCreate(&ev0));
        MAG_CUDA(cudaEventCreate(&ev1));
        MAG_TRY(alloc((void**)&d_chains, sizeof(ChainInfo) * n));
        const long nchunk = vpad / MAG_CHUNK;
        MAG_TRY(alloc((void**)&d_c2c, sizeof(uint16_t) * nchunk));
        std::vector<uint16_t> c2c(nchunk, 0);
        for (int c = 0; c < n; c++)
            for (long k = hc[c].off / MAG_CHUNK; k < (hc[c].off + hc[c].V + MAG_CHUNK - 1) / MAG_CHUNK; k++)
                c2c[k] = (uint16_t)c;
        // on the context's stream (a pageable cudaMemcpy may return before its DMA lands, and the
        // non-blocking stream would not wait for it); the sync at the end of init covers them
        MAG_CUDA(cudaMemcpyAsync(d_chains, hc.data(), sizeof(ChainInfo) * n, cudaMemcpyHostToDevice, stream));
        MAG_CUDA(cudaMemcpyAsync(d_c2c, c2c.data(), sizeof(uint16_t) * nchunk, cudaMemcpyHostToDevice, stream));
        MAG_TRY(alloc((void**)&d_stream_index, sizeof(unsigned long long) * n));
        std::vector<unsigned long long> sidx(n);
        for (int c = 0; c < n; c++) sidx[c] = (unsigned long long)c;
        MAG_CUDA(cudaMemcpyAsync(d_stream_index, sidx.data(), sizeof(unsigned long long) * n,
                                 cudaMemcpyHostToDevice, stream));
        h_stream_index = sidx;
        geom = DevGeom{d_chains, d_c2c, vpad, n, d_stream_index, 0, 0, 0};

        MAG_TRY(alloc_links(U));
        MAG_TRY(alloc_links(Ubak));
        MAG_TRY(alloc_alg(P));
        if (mixed) {
            MAG_TRY(alloc_links(U32));
            MAG_TRY(alloc_links(Uaux32));
            MAG_TRY(alloc_alg(F32));
            MAG_TRY(alloc_stout(st32, true));
            MAG_TRY(alloc_stout(st64, false));  // FP64 forward smearing for the Hamiltonian
            MAG_TRY(alloc_alg(F));              // FP64 force for single-call API use
            if (iwasaki) MAG_TRY(alloc_links(W32));
        } else {
            MAG_TRY(alloc_links(Uaux));
            MAG_TRY(alloc_alg(F));
            MAG_TRY(alloc_stout(st64, true));
            if (iwasaki) MAG_TRY(alloc_links(W64));
        }
        MAG_TRY(alloc((void**)&partial, sizeof(dd2) * 2 * (nchunk + 1)));
        MAG_TRY(alloc((void**)&sums, sizeof(dd2) * NUM_SLOTS * n));
        MAG_TRY(alloc((void**)&cstate, sizeof(ChainState) * n));
        MAG_TRY(alloc((void**)&reunit, sizeof(unsigned long long) * n));
        MAG_TRY(alloc((void**)&rec, sizeof(TrajRecord) * n));
        MAG_TRY(alloc((void**)&hist, sizeof(TrajRecord) * n * kHistCap));
        MAG_TRY(alloc((void**)&hist_base, sizeof(long long)));
        MAG_TRY(alloc((void**)&traj_counter, sizeof(long long)));
        MAG_TRY(alloc((void**)&tmp_counter, sizeof(long long)));
        MAG_TRY(alloc((void**)&d_uniform, sizeof(double) * n));
        MAG_TRY(alloc((void**)&staging, sizeof(double) * 72 * (size_t)max_v));
        MAG_CUDA(cudaMemsetAsync(cstate, 0, sizeof(ChainState) * n, stream));
        MAG_CUDA(cudaMemsetAsync(reunit, 0, sizeof(unsigned long long) * n, stream));
        MAG_CUDA(cudaMemsetAsync(traj_counter, 0, sizeof(long long), stream));
        MAG_CUDA(cudaMemsetAsync(hist_base, 0, sizeof(long long), stream));
        launch_cold_start(geom, U, stream);
        MAG_TRY(refresh_copy());
        return sync("context init");
    }

    int refresh_copy() {
        if (mixed) launch_copy_to_float(geom, U, U32, stream);
        return check("refresh fp32 links");
    }

    // ----------------------------------------------------------- force
    // register-cap variant per kernel family and precision ([0] double, [1] float)
    int tune[KF_COUNT][2] = {};
    double tune_ms[KF_COUNT][2][kNumVariants] = {};  // the tuner's times per variant (0: not timed)
    bool tuned = false;
    // families with direction-split variants (the others have the register caps only)
    static int variants_of(KernelFamily f) {
        return (f == KF_FORCE || f == KF_STAPLE || f == KF_STOUT_CHAIN) ? kNumVariants : kNumRegVariants;
    }
    template <typename T>
    int var(KernelFamily f) const {
        return tune[f][sizeof(T) == 8 ? 0 : 1];
    }

    // double links of the field whose staples are being summed (Iwasaki only)
    LinkPlanes<double> W64{nullptr, 0};
    LinkPlanes<float> W32{nullptr, 0};
    template <typename T>
    LinkPlanes<T> wbuf() const {
        if constexpr (sizeof(T) == 8) return W64;
        else return W32;
    }

    // A sharded context exchanges halos (hx) after every launch whose output a
    // later kernel reads across the shard boundary: the links whose force is
    // taken, each smeared level, the double links and Lambda of each level.
    template <typename T>
    void force_eval(LinkPlanes<T> Uin, AlgPlanes<T> Fout, StoutBufs<T>& b) {
        hx(Uin);
        if (p.n_stout == 0) {
            if (iwasaki) {
                launch_double_link<T>(geom, Uin, wbuf<T>(), stream);
                hx(wbuf<T>());
            }
            launch_force<T>(geom, Uin, wbuf<T>(), Fout, iwasaki, var<T>(KF_FORCE), stream);
        } else {
            LinkPlanes<T> cur = Uin;
            for (int k = 0; k < p.n_stout; k++) {
                launch_stout_forward<T>(geom, cur, b.lv[k], b.Q[k], var<T>(KF_STOUT_FWD), stream);
                cur = b.lv[k];
                hx(cur);
            }
            if (iwasaki) {
                launch_double_link<T>(geom, cur, wbuf<T>(), stream);
                hx(wbuf<T>());
            }
            launch_staple_dagger<T>(geom, cur, wbuf<T>(), b.za, iwasaki, var<T>(KF_STAPLE), stream);
            for (int k = p.n_stout - 1; k >= 0; k--) {
                LinkPlanes<T> ul = k == 0 ? Uin : b.lv[k - 1];
                launch_stout_lambda<T>(geom, ul, b.Q[k], b.za, b.lam, b.zp, var<T>(KF_STOUT_LAMBDA), stream);
                hx(b.lam);
                if (k == 0) launch_stout_chain_force<T>(geom, ul, b.lam, b.zp, Fout, var<T>(KF_STOUT_CHAIN), stream);
                else launch_stout_chain<T>(geom, ul, b.lam, b.zp, b.za, var<T>(KF_STOUT_CHAIN), stream);
            }
        }
        if (any_mag) launch_constraint_fixup<T>(geom, Uin, Fout, stream);
    }

    // smeared FP64 links for the Hamiltonian (the thin links when n_stout = 0)
    LinkPlanes<double> smear64() {
        LinkPlanes<double> cur = U;
        hx(cur);
        for (int k = 0; k < p.n_stout; k++) {
            launch_stout_forward<double>(geom, cur, st64.lv[k], st64.Q[k], var<double>(KF_STOUT_FWD), stream);
            cur = st64.lv[k];
            hx(cur);
        }
        return cur;
    }

    // one launch of a kernel family on the live buffers of precision T
    template <typename T>
    void launch_one(KernelFamily f, int v, StoutBufs<T>& b, LinkPlanes<T> Uin, AlgPlanes<T> Fo, LinkPlanes<T> zs) {
        const int L = p.n_stout;
        switch (f) {
            case KF_FORCE: launch_force<T>(geom, Uin, wbuf<T>(), Fo, iwasaki, v, stream); break;
            case KF_STAPLE:
                launch_staple_dagger<T>(geom, L ? b.lv[L - 1] : Uin, wbuf<T>(), L ? b.za : zs, iwasaki, v, stream);
                break;
            case KF_STOUT_FWD: launch_stout_forward<T>(geom, Uin, b.lv[0], b.Q[0], v, stream); break;
            case KF_STOUT_LAMBDA: launch_stout_lambda<T>(geom, Uin, b.Q[0], b.za, b.lam, b.zp, v, stream); break;
            case KF_STOUT_CHAIN: launch_stout_chain<T>(geom, Uin, b.lam, b.zp, b.za, v, stream); break;
            default: break;
        }
    }

    template <typename T>
    int time_one(KernelFamily f, int v, int reps, StoutBufs<T>& b, LinkPlanes<T> Uin, AlgPlanes<T> Fo,
                 LinkPlanes<T> zs, double* ms) {
        launch_one<T>(f, v, b, Uin, Fo, zs);
        MAG_CUDA(cudaEventRecord(ev0, stream));
        for (int i = 0; i < reps; i++) launch_one<T>(f, v, b, Uin, Fo, zs);
        MAG_CUDA(cudaEventRecord(ev1, stream));
        MAG_TRY(sync("time kernel"));
        float t = 0.f;
        MAG_CUDA(cudaEventElapsedTime(&t, ev0, ev1));
        *ms = t / reps;
        return MAG_OK;
    }

    // The tuner: time every register-cap variant of every kernel family the
    // integrator uses, on live data, and keep the fastest.  Variants compute
    // identical results (same instructions, different register allocation).
    template <typename T>
    int tune_precision(int reps, StoutBufs<T>& b, LinkPlanes<T> Uin, AlgPlanes<T> Fo, LinkPlanes<T> zs) {
        force_eval<T>(Uin, Fo, b);
        std::vector<KernelFamily> fams;
        if (p.n_stout == 0) fams = {KF_FORCE};
        else fams = {KF_STAPLE, KF_STOUT_FWD, KF_STOUT_LAMBDA, KF_STOUT_CHAIN};
        // Every variant is timed (the report shows them all), but the choice is made among the
        // one-thread-per-link register caps only: those compute bit-identical results, so a run does not
        // depend on timing noise.  The direction-split shapes add their parts in another order (results
        // differ by rounding) and measured slower at every lattice size tried; mag_set_kernel_variant
        // selects one explicitly.
        const int pi = sizeof(T) == 8 ? 0 : 1;
        for (KernelFamily f : fams) {
            double best = 1e300;
            int bv = 0;
            for (int v = 0; v < variants_of(f); v++) {
                double ms = 0.0;
                MAG_TRY(time_one<T>(f, v, reps, b, Uin, Fo, zs, &ms));
                tune_ms[f][pi][v] = ms;
                if (v < kNumRegVariants && ms < best) {
                    best = ms;
                    bv = v;
                }
            }
            tune[f][pi] = bv;
        }
        return MAG_OK;
    }

    // Block traversal order of the link kernels for a single lattice: raster,
    // or (x2, x3) rows in T x T tiles (T = 2, 4), timed on whole force
    // evaluations; every order computes bit-identical results.
    double tile_time_ms[3] = {};
    template <typename T>
    int tune_order(int reps, StoutBufs<T>& b, LinkPlanes<T> Uin, AlgPlanes<T> Fo) {
        geom.tile = 0;
        const ChainInfo& c = hc[0];
        const long row = (long)c.L[0] * c.L[1];
        if (nchain != 1 || row % kForceBlockSites || c.V % MAG_CHUNK) return MAG_OK;
        double best = 1e300;
        int bt = 0;
        for (int k = 0; k < 3; k++) {
            const int tl = k == 0 ? 0 : 2 * k;  // 0, 2, 4
            if (tl && (c.L[2] % tl || c.L[3] % tl)) continue;
            geom.tile = tl;
            geom.gpr = (int)(row / kForceBlockSites);
            geom.L2 = c.L[2];
            force_eval<T>(Uin, Fo, b);
            MAG_CUDA(cudaEventRecord(ev0, stream));
            for (int i = 0; i < reps; i++) force_eval<T>(Uin, Fo, b);
            MAG_CUDA(cudaEventRecord(ev1, stream));
            MAG_TRY(sync("tune order"));
            float t = 0.f;
            MAG_CUDA(cudaEventElapsedTime(&t, ev0, ev1));
            tile_time_ms[k] = t / reps;
            if (t < best) {
                best = t;
                bt = tl;
            }
        }
        geom.tile = bt;
        return MAG_OK;
    }

    int autotune(int reps) {
        if (mixed) {
            MAG_TRY(tune_precision<float>(reps, st32, U32, F32, Uaux32));
            if (p.n_stout > 0) {
                // the FP64 forward smearing of the Hamiltonian
                double best = 1e300;
                for (int v = 0; v < kNumRegVariants; v++) {
                    double ms = 0.0;
                    StoutBufs<double> b = st64;
                    MAG_TRY(time_one<double>(KF_STOUT_FWD, v, reps, b, U, F, Ubak, &ms));
                    tune_ms[KF_STOUT_FWD][0][v] = ms;
                    if (ms < best) {
                        best = ms;
                        tune[KF_STOUT_FWD][0] = v;
                    }
                }
            }
        } else {
            MAG_TRY(tune_precision<double>(reps, st64, U, F, Uaux));
        }
        if (!halo) {
            if (mixed) MAG_TRY(tune_order<float>(reps, st32, U32, F32));
            else MAG_TRY(tune_order<double>(reps, st64, U, F));
        }
        tuned = true;
        return MAG_OK;
    }
    int ensure_tuned() { return tuned ? MAG_OK : autotune(3); }

    void hamiltonian_sums(bool is_new) {
        launch_kinetic_sum(geom, P, partial, sums, is_new ? SLOT_KIN_NEW : SLOT_KIN_OLD, stream);
        LinkPlanes<double> top = smear64();
        launch_action_sums<double>(geom, top, true, partial, sums, is_new ? SLOT_PLAQ_NEW : SLOT_PLAQ_OLD,
                                   is_new ? SLOT_RECT_NEW : SLOT_RECT_OLD, stream);
        if (is_new) hreduce({SLOT_KIN_NEW, SLOT_PLAQ_NEW, SLOT_RECT_NEW}, true);
        else hreduce({SLOT_KIN_OLD, SLOT_PLAQ_OLD, SLOT_RECT_OLD}, false);
    }

    // ------------------------------------------------------- integrator
    template <typename T>
    void integrate_t(LinkPlanes<T> Ut, LinkPlanes<T> Ua, AlgPlanes<T> Fw, StoutBufs<T>& b) {
        const double dt = p.tau / p.n_steps;
        LinkPlanes<float> copy = mixed ? U32 : LinkPlanes<float>{nullptr, 0};
        auto master = [&](double eps) { launch_evolve<double, double>(geom, U, U, P, eps, copy, stream); };
        if (p.integrator == MAG_INT_LEAPFROG) {
            master(dt / 2.);
            for (int i = 0; i < p.n_steps; i++) {
                force_eval<T>(Ut, Fw, b);
                launch_kick<T>(geom, P, Fw, dt, stream);
                master(i < p.n_steps - 1 ? dt : dt / 2.);
            }
            return;
        }
        const double alpha = (3. - std::sqrt(3.)) * dt / 6.;
        const double beta = dt / std::sqrt(3.);
        const double gamma = (2. - std::sqrt(3.)) * dt * dt / 12.;
        auto fg_kick = [&]() {
            force_eval<T>(Ut, Fw, b);
            launch_evolve<T, T>(geom, Ut, Ua, Fw, gamma, LinkPlanes<float>{nullptr, 0}, stream);
            force_eval<T>(Ua, Fw, b);
            launch_kick<T>(geom, P, Fw, 0.5 * dt, stream);
        };
        master(alpha);
        for (int i = 0; i < p.n_steps; i++) {
            fg_kick();
            master(beta);
            fg_kick();
            master(i < p.n_steps - 1 ? 2. * alpha : alpha);
        }
    }

    int integrate() {
        if (mixed) integrate_t<float>(U32, Uaux32, F32, st32);
        else integrate_t<double>(U, Uaux, F, st64);
        cudaMemsetAsync(reunit, 0, sizeof(unsigned long long) * nchain, stream);
        if (p.integrator != MAG_INT_LEAPFROG)
            launch_reunitarize(geom, U, mixed ? U32 : LinkPlanes<float>{nullptr, 0}, reunit, stream);
        return check("integrate");
    }

    // one trajectory as a fixed launch sequence
    int trajectory_body(bool refresh) {
        if (refresh) launch_momenta(geom, P, p.seed, traj_counter, stream);
        launch_link_copy(geom, U, Ubak, stream);
        hamiltonian_sums(false);
        const int ri = integrate();
        if (ri != MAG_OK && !halo) return ri;  // a shard keeps meeting the others at the exchange points
        hamiltonian_sums(true);
        AcceptArgs a;
        a.metropolis = p.accept == MAG_ACCEPT_METROPOLIS ? 1 : 0;
        a.action_iwasaki = iwasaki ? 1 : 0;
        a.e_max = p.e_max;
        a.n_forced = p.n_forced_accept;
        a.uniform_override = uniform_override ? d_uniform : nullptr;
        a.seed = p.seed;
        launch_accept(geom, a, sums, cstate, reunit, rec, traj_counter, stream);
        launch_restore_rejected(geom, Ubak, U, mixed ? U32 : LinkPlanes<float>{nullptr, 0}, cstate, stream);
        hx(U);
        launch_action_sums<double>(geom, U, false, partial, sums, SLOT_PLAQ_THIN, SLOT_RECT_THIN, stream);
        hreduce({SLOT_PLAQ_THIN, SLOT_RECT_THIN}, false);
        launch_record_plaquette(geom, sums, rec, hist, hist_base, kHistCap, traj_counter, stream);
        if (halo_rc != MAG_OK) return halo_rc;
        if (ri != MAG_OK) return ri;
        return check("trajectory");
    }

    int build_graph() {
        if (graph) return MAG_OK;
        MAG_TRY(ensure_tuned());
        cudaGraph_t g;
        MAG_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int r = trajectory_body(true);
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (r != MAG_OK) return r;
        if (e != cudaSuccess) return fail(MAG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        cudaGraphGetNodes(g, nodes.data(), &nn);
        graph_kernels = 0;
        for (size_t k = 0; k < nn; k++) {
            cudaGraphNodeType t;
            cudaGraphNodeGetType(nodes[k], &t);
            if (t == cudaGraphNodeTypeKernel) graph_kernels++;
        }
        e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(MAG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        return MAG_OK;
    }

    static void to_result(const TrajRecord& r, mag_traj_result* o) {
        o->h_old = r.h_old; o->h_new = r.h_new; o->delta_h = r.delta_h;
        o->kinetic_old = r.kin_old; o->kinetic_new = r.kin_new;
        o->action_old = r.pot_old; o->action_new = r.pot_new;
        o->plaq_sum_old = r.plaq_old; o->plaq_sum_new = r.plaq_new;
        o->rect_sum_old = r.rect_old; o->rect_sum_new = r.rect_new;
        o->uniform = r.uniform;
        o->demon[0] = r.demon0; o->demon[1] = r.demon1;
        o->reunit_maxdev = r.reunit_maxdev;
        o->avg_plaquette = r.avg_plaquette;
        o->accept = r.accept;
        o->traj = r.traj;
    }

    // lazily sized measurement buffers (Wilson loops, closed paths)
    dd2* wl_partial = nullptr;
    dd2* wl_out = nullptr;
    cplx<double>* wl_lines = nullptr;
    int* d_paths = nullptr;
    int wl_rmax = 0, wl_tmax = 0;
    const int max_path_ints = 4096;

    void free_one(void* p) {
        if (!p) return;
        for (size_t k = 0; k < allocs.size(); k++)
            if (allocs[k] == p) {
                allocs.erase(allocs.begin() + k);
                break;
            }
        cudaFree(p);
    }

    // Rmax x Tmax planar loops need Rmax + 2 single-direction line planes
    int ensure_meas(int Rmax, int Tmax, bool lines) {
        if (!d_paths) MAG_TRY(alloc((void**)&d_paths, sizeof(int) * max_path_ints));
        const bool grow = !wl_partial || Rmax > wl_rmax || Tmax > wl_tmax || (lines && !wl_lines);
        if (!grow) return MAG_OK;
        cudaStreamSynchronize(stream);
        Rmax = std::max(Rmax, wl_rmax);
        Tmax = std::max(Tmax, wl_tmax);
        const size_t nb = (size_t)(vpad / MAG_CHUNK) + 1;
        free_one(wl_partial);
        free_one(wl_out);
        free_one(wl_lines);
        wl_lines = nullptr;
        MAG_TRY(alloc((void**)&wl_partial, sizeof(dd2) * nb * Rmax));
        MAG_TRY(alloc((void**)&wl_out, sizeof(dd2) * ((size_t)3 * Tmax * nchain * Rmax + nchain)));
        if (lines) MAG_TRY(alloc((void**)&wl_lines, sizeof(cplx<double>) * 9 * (size_t)vpad * (Rmax + 2)));
        wl_rmax = Rmax;
        wl_tmax = Tmax;
        return MAG_OK;
    }

    int chain_ok(int c) {
        if (c < 0 || c >= nchain) return fail(MAG_ERR_ARG, "chain index out of range");
        return MAG_OK;
    }

    // read per-chain double-double sums back to the host
    int read_sums(std::vector<dd2>& out) {
        out.resize((size_t)NUM_SLOTS * nchain);
        MAG_CUDA(cudaMemcpyAsync(out.data(), sums, sizeof(dd2) * out.size(), cudaMemcpyDeviceToHost, stream));
        return sync("read sums");
    }

    hdd action_value(int c, dd2 plaq, dd2 rect) const {
        const ChainInfo& ci = hc[c];
        hdd t = iwasaki ? h_add(h_mul(h_neg(hdd{plaq.hi, plaq.lo}), ci.c0), h_mul(h_neg(hdd{rect.hi, rect.lo}), ci.c1))
                        : h_neg(hdd{plaq.hi, plaq.lo});
        return h_mul(t, ci.beta / 3.0);
    }
};

