// mag_api.cu -- C++ host driver and C ABI of libmag_b200.so.
//
// The context owns every device buffer and one stream.  The integrator is the
// force-gradient scheme of field-hmc.h:525-567 (or the leapfrog of :569-587)
// written as a fixed launch sequence with device-resident scalars, so one HMC
// trajectory (momenta, H_old, integration, reunitarisation, H_new, accept,
// restore, record) replays as a single CUDA graph with no host round trip.
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

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
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
hdd h_two_sum(double a, double b) {
    const double s = a + b, bp = s - a;
    return hdd{s, (a - (s - bp)) + (b - bp)};
}
hdd h_add(hdd a, hdd b) {
    hdd s = h_two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return h_two_sum(s.hi, s.lo);
}
hdd h_mul(hdd a, double b) {
    const double p = a.hi * b;
    const double e = std::fma(a.hi, b, -p);
    return h_two_sum(p, e + a.lo * b);
}
hdd h_neg(hdd a) { return hdd{-a.hi, -a.lo}; }

}  // namespace

namespace magb {
// lets the allocation-free entry point (noalloc.cu) report through mag_last_error()
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace magb

struct mag_ctx;
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

// ======================================================================= C ABI
namespace {

// a device buffer released on every return path
struct DeviceBuffer {
    void* p = nullptr;
    ~DeviceBuffer() {
        if (p) cudaFree(p);
    }
};

// n 3x3 complex matrices (144 bytes each) in from the host, `run` on the device, n out
template <typename Run>
int matrix_op(const char* name, const double* const* in, int nin, int64_t n, double* out, Run run) {
    for (int k = 0; k < nin; k++)
        if (!in[k]) return fail(MAG_ERR_ARG, std::string(name) + ": null input");
    if (!out || n < 0) return fail(MAG_ERR_ARG, std::string(name) + ": bad argument");
    if (n == 0) return MAG_OK;
    const size_t bytes = (size_t)n * 144;
    DeviceBuffer din[3], dout;
    for (int k = 0; k < nin; k++) {
        MAG_CUDA(cudaMalloc(&din[k].p, bytes));
        MAG_CUDA(cudaMemcpy(din[k].p, in[k], bytes, cudaMemcpyHostToDevice));
    }
    MAG_CUDA(cudaMalloc(&dout.p, bytes));
    run((const double*)din[0].p, (const double*)din[1].p, (const double*)din[2].p, (double*)dout.p);
    MAG_CUDA(cudaGetLastError());
    MAG_CUDA(cudaMemcpy(out, dout.p, bytes, cudaMemcpyDeviceToHost));
    return MAG_OK;
}

}  // namespace

extern "C" {

const char* mag_last_error(void) { return g_last_error.c_str(); }

int mag_ensemble_create(const mag_params* p, int n, mag_ctx** out) {
    if (!p || !out || n < 1 || n > 1024) return fail(MAG_ERR_ARG, "mag_ensemble_create: bad arguments");
    *out = nullptr;
    mag_ctx* c = new mag_ctx();
    const int r = c->init(p, n);
    if (r != MAG_OK) {
        delete c;
        return r;
    }
    *out = c;
    return MAG_OK;
}

int mag_ctx_create(const mag_params* p, mag_ctx** out) { return mag_ensemble_create(p, 1, out); }

int mag_ctx_destroy(mag_ctx* ctx) {
    if (!ctx) return MAG_ERR_ARG;
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
    return MAG_OK;
}

int mag_ctx_num_chains(const mag_ctx* ctx, int* n) {
    if (!ctx || !n) return MAG_ERR_ARG;
    *n = ctx->nchain;
    return MAG_OK;
}

int mag_ctx_device_bytes(const mag_ctx* ctx, size_t* bytes) {
    if (!ctx || !bytes) return MAG_ERR_ARG;
    *bytes = ctx->bytes;
    return MAG_OK;
}

int mag_gauge_set(mag_ctx* ctx, int chain, const double* host) {
    if (!ctx || !host) return fail(MAG_ERR_ARG, "mag_gauge_set: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    MAG_CUDA(cudaMemcpyAsync(ctx->staging, host, sizeof(double) * 72 * (size_t)ci.V, cudaMemcpyHostToDevice,
                             ctx->stream));
    launch_aos_to_links(ctx->staging, ci.off, ci.V, ctx->U, ctx->vpad, ctx->stream);
    MAG_TRY(ctx->refresh_copy());
    return ctx->sync("mag_gauge_set");
}

int mag_gauge_get(mag_ctx* ctx, int chain, double* host) {
    if (!ctx || !host) return fail(MAG_ERR_ARG, "mag_gauge_get: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    launch_links_to_aos(ctx->U, ci.off, ci.V, ctx->staging, ctx->stream);
    MAG_CUDA(cudaMemcpyAsync(host, ctx->staging, sizeof(double) * 72 * (size_t)ci.V, cudaMemcpyDeviceToHost,
                             ctx->stream));
    return ctx->sync("mag_gauge_get");
}

int mag_gauge_hot_start(mag_ctx* ctx, uint64_t seed) {
    if (!ctx) return MAG_ERR_ARG;
    launch_hot_start(ctx->geom, ctx->U, seed, ctx->stream);
    MAG_TRY(ctx->refresh_copy());
    return ctx->sync("mag_gauge_hot_start");
}

int mag_gauge_cold_start(mag_ctx* ctx) {
    if (!ctx) return MAG_ERR_ARG;
    launch_cold_start(ctx->geom, ctx->U, ctx->stream);
    MAG_TRY(ctx->refresh_copy());
    return ctx->sync("mag_gauge_cold_start");
}

int mag_momentum_set(mag_ctx* ctx, int chain, const double* host) {
    if (!ctx || !host) return fail(MAG_ERR_ARG, "mag_momentum_set: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    MAG_CUDA(cudaMemcpyAsync(ctx->staging, host, sizeof(double) * 72 * (size_t)ci.V, cudaMemcpyHostToDevice,
                             ctx->stream));
    launch_aos_to_alg<double>(ctx->staging, ci.off, ci.V, ctx->P, ctx->stream);
    return ctx->sync("mag_momentum_set");
}

int mag_momentum_get(mag_ctx* ctx, int chain, double* host) {
    if (!ctx || !host) return fail(MAG_ERR_ARG, "mag_momentum_get: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    launch_alg_to_aos<double>(ctx->P, ci.off, ci.V, ctx->staging, ctx->stream);
    MAG_CUDA(cudaMemcpyAsync(host, ctx->staging, sizeof(double) * 72 * (size_t)ci.V, cudaMemcpyDeviceToHost,
                             ctx->stream));
    return ctx->sync("mag_momentum_get");
}

int mag_momentum_refresh(mag_ctx* ctx, uint64_t traj) {
    if (!ctx) return MAG_ERR_ARG;
    const long long t = (long long)traj;
    MAG_CUDA(cudaMemcpyAsync(ctx->tmp_counter, &t, sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    launch_momenta(ctx->geom, ctx->P, ctx->p.seed, ctx->tmp_counter, ctx->stream);
    return ctx->sync("mag_momentum_refresh");
}

int mag_uniforms_set(mag_ctx* ctx, const double* u) {
    if (!ctx) return MAG_ERR_ARG;
    const bool was = ctx->uniform_override;
    if (!u) {
        ctx->uniform_override = false;
    } else {
        MAG_CUDA(cudaMemcpyAsync(ctx->d_uniform, u, sizeof(double) * ctx->nchain, cudaMemcpyHostToDevice,
                                 ctx->stream));
        ctx->uniform_override = true;
    }
    if (was != ctx->uniform_override && ctx->graph) {
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
    return ctx->sync("mag_uniforms_set");
}

int mag_gauge_force(mag_ctx* ctx, int chain, double* host) {
    if (!ctx || !host) return fail(MAG_ERR_ARG, "mag_gauge_force: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    if (ctx->mixed) {
        ctx->force_eval<float>(ctx->U32, ctx->F32, ctx->st32);
        launch_alg_to_aos<float>(ctx->F32, ci.off, ci.V, ctx->staging, ctx->stream);
    } else {
        ctx->force_eval<double>(ctx->U, ctx->F, ctx->st64);
        launch_alg_to_aos<double>(ctx->F, ci.off, ci.V, ctx->staging, ctx->stream);
    }
    MAG_TRY(ctx->check("mag_gauge_force"));
    MAG_CUDA(cudaMemcpyAsync(host, ctx->staging, sizeof(double) * 72 * (size_t)ci.V, cudaMemcpyDeviceToHost,
                             ctx->stream));
    return ctx->sync("mag_gauge_force");
}

int mag_staple(mag_ctx* ctx, int chain, double* host) {
    if (!ctx || !host) return fail(MAG_ERR_ARG, "mag_staple: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    if (ctx->mixed) {
        LinkPlanes<float> cur = ctx->U32;
        for (int k = 0; k < ctx->p.n_stout; k++) {
            launch_stout_forward<float>(ctx->geom, cur, ctx->st32.lv[k], ctx->st32.Q[k],
                                        ctx->var<float>(KF_STOUT_FWD), ctx->stream);
            cur = ctx->st32.lv[k];
        }
        LinkPlanes<float> z = ctx->p.n_stout ? ctx->st32.za : ctx->Uaux32;
        if (ctx->iwasaki) launch_double_link<float>(ctx->geom, cur, ctx->W32, ctx->stream);
        launch_staple_dagger<float>(ctx->geom, cur, ctx->W32, z, ctx->iwasaki, ctx->var<float>(KF_STAPLE),
                                    ctx->stream);
        launch_links_to_aos_t<float>(z, ci.off, ci.V, ctx->staging, ctx->stream);
    } else {
        LinkPlanes<double> cur = ctx->smear64();
        LinkPlanes<double> z = ctx->p.n_stout ? ctx->st64.za : ctx->Uaux;
        if (ctx->iwasaki) launch_double_link<double>(ctx->geom, cur, ctx->W64, ctx->stream);
        launch_staple_dagger<double>(ctx->geom, cur, ctx->W64, z, ctx->iwasaki, ctx->var<double>(KF_STAPLE),
                                     ctx->stream);
        launch_links_to_aos_t<double>(z, ci.off, ci.V, ctx->staging, ctx->stream);
    }
    MAG_TRY(ctx->check("mag_staple"));
    MAG_CUDA(cudaMemcpyAsync(host, ctx->staging, sizeof(double) * 72 * (size_t)ci.V, cudaMemcpyDeviceToHost,
                             ctx->stream));
    return ctx->sync("mag_staple");
}

int mag_action(mag_ctx* ctx, int chain, double* plaq, double* rect, double* action) {
    if (!ctx) return MAG_ERR_ARG;
    MAG_TRY(ctx->chain_ok(chain));
    LinkPlanes<double> top = ctx->smear64();
    launch_action_sums<double>(ctx->geom, top, true, ctx->partial, ctx->sums, SLOT_PLAQ_THIN, SLOT_RECT_THIN,
                               ctx->stream);
    MAG_TRY(ctx->check("mag_action"));
    std::vector<dd2> s;
    MAG_TRY(ctx->read_sums(s));
    const dd2 pl = s[chain * NUM_SLOTS + SLOT_PLAQ_THIN], re = s[chain * NUM_SLOTS + SLOT_RECT_THIN];
    if (plaq) *plaq = pl.hi + pl.lo;
    if (rect) *rect = re.hi + re.lo;
    const hdd a = ctx->action_value(chain, pl, re);
    if (action) *action = a.hi + a.lo;
    return MAG_OK;
}

int mag_plaquette(mag_ctx* ctx, int chain, double* avg) {
    if (!ctx || !avg) return MAG_ERR_ARG;
    MAG_TRY(ctx->chain_ok(chain));
    launch_action_sums<double>(ctx->geom, ctx->U, false, ctx->partial, ctx->sums, SLOT_SCRATCH, SLOT_SCRATCH,
                               ctx->stream);
    MAG_TRY(ctx->check("mag_plaquette"));
    std::vector<dd2> s;
    MAG_TRY(ctx->read_sums(s));
    const dd2 pl = s[chain * NUM_SLOTS + SLOT_SCRATCH];
    *avg = (pl.hi + pl.lo) / (18.0 * ctx->hc[chain].V);
    return MAG_OK;
}

int mag_kinetic(mag_ctx* ctx, int chain, double* kin) {
    if (!ctx || !kin) return MAG_ERR_ARG;
    MAG_TRY(ctx->chain_ok(chain));
    launch_kinetic_sum(ctx->geom, ctx->P, ctx->partial, ctx->sums, SLOT_SCRATCH, ctx->stream);
    MAG_TRY(ctx->check("mag_kinetic"));
    std::vector<dd2> s;
    MAG_TRY(ctx->read_sums(s));
    const dd2 k = s[chain * NUM_SLOTS + SLOT_SCRATCH];
    *kin = k.hi + k.lo;
    return MAG_OK;
}

int mag_hamiltonian(mag_ctx* ctx, int chain, double out[3]) {
    if (!ctx || !out) return MAG_ERR_ARG;
    MAG_TRY(ctx->chain_ok(chain));
    ctx->hamiltonian_sums(false);
    MAG_TRY(ctx->check("mag_hamiltonian"));
    std::vector<dd2> s;
    MAG_TRY(ctx->read_sums(s));
    const dd2* S = s.data() + chain * NUM_SLOTS;
    const hdd a = ctx->action_value(chain, S[SLOT_PLAQ_OLD], S[SLOT_RECT_OLD]);
    const hdd k = hdd{S[SLOT_KIN_OLD].hi, S[SLOT_KIN_OLD].lo};
    const hdd h = h_add(a, k);
    out[0] = h.hi + h.lo;
    out[1] = k.hi + k.lo;
    out[2] = a.hi + a.lo;
    return MAG_OK;
}

int mag_evolve_gauge(mag_ctx* ctx, double eps) {
    if (!ctx) return MAG_ERR_ARG;
    launch_evolve<double, double>(ctx->geom, ctx->U, ctx->U, ctx->P, eps,
                                  ctx->mixed ? ctx->U32 : LinkPlanes<float>{nullptr, 0}, ctx->stream);
    return ctx->sync("mag_evolve_gauge");
}

int mag_evolve_gauge_src(mag_ctx* ctx, double eps, int src) {
    if (!ctx) return MAG_ERR_ARG;
    if (src == MAG_SRC_MOMENTA) return mag_evolve_gauge(ctx, eps);
    if (src != MAG_SRC_FORCE) return fail(MAG_ERR_ARG, "mag_evolve_gauge_src: src must be MAG_SRC_MOMENTA or MAG_SRC_FORCE");
    // the force-gradient step's link update U <- exp(i eps F(U)) U (field-hmc.h:497-503)
    if (ctx->mixed) {
        ctx->force_eval<float>(ctx->U32, ctx->F32, ctx->st32);
        launch_evolve<double, float>(ctx->geom, ctx->U, ctx->U, ctx->F32, eps, ctx->U32, ctx->stream);
    } else {
        ctx->force_eval<double>(ctx->U, ctx->F, ctx->st64);
        launch_evolve<double, double>(ctx->geom, ctx->U, ctx->U, ctx->F, eps, LinkPlanes<float>{nullptr, 0},
                                      ctx->stream);
    }
    return ctx->sync("mag_evolve_gauge_src");
}

int mag_stout_forward(mag_ctx* ctx, int chain, int level, double* host_aos) {
    return mag_stout_level(ctx, chain, level, host_aos);
}

int mag_stout_force(mag_ctx* ctx, int chain, double* host_force_aos) {
    if (ctx && ctx->p.n_stout < 1) return fail(MAG_ERR_STATE, "mag_stout_force: context has no stout levels");
    return mag_gauge_force(ctx, chain, host_force_aos);
}

int mag_evolve_momentum(mag_ctx* ctx, double eps) {
    if (!ctx) return MAG_ERR_ARG;
    if (ctx->mixed) {
        ctx->force_eval<float>(ctx->U32, ctx->F32, ctx->st32);
        launch_kick<float>(ctx->geom, ctx->P, ctx->F32, eps, ctx->stream);
    } else {
        ctx->force_eval<double>(ctx->U, ctx->F, ctx->st64);
        launch_kick<double>(ctx->geom, ctx->P, ctx->F, eps, ctx->stream);
    }
    return ctx->sync("mag_evolve_momentum");
}

int mag_reunitarize(mag_ctx* ctx, double* maxdev) {
    if (!ctx) return MAG_ERR_ARG;
    MAG_CUDA(cudaMemsetAsync(ctx->reunit, 0, sizeof(unsigned long long) * ctx->nchain, ctx->stream));
    launch_reunitarize(ctx->geom, ctx->U, ctx->mixed ? ctx->U32 : LinkPlanes<float>{nullptr, 0}, ctx->reunit,
                       ctx->stream);
    MAG_TRY(ctx->check("mag_reunitarize"));
    std::vector<unsigned long long> bits(ctx->nchain);
    MAG_CUDA(cudaMemcpyAsync(bits.data(), ctx->reunit, sizeof(unsigned long long) * ctx->nchain,
                             cudaMemcpyDeviceToHost, ctx->stream));
    MAG_TRY(ctx->sync("mag_reunitarize"));
    if (maxdev)
        for (int c = 0; c < ctx->nchain; c++) std::memcpy(&maxdev[c], &bits[c], sizeof(double));
    return MAG_OK;
}

int mag_stout_level(mag_ctx* ctx, int chain, int level, double* host) {
    if (!ctx || !host) return MAG_ERR_ARG;
    MAG_TRY(ctx->chain_ok(chain));
    if (level < 0 || level > ctx->p.n_stout) return fail(MAG_ERR_ARG, "stout level out of range");
    const ChainInfo& ci = ctx->hc[chain];
    ctx->smear64();
    LinkPlanes<double> l = level == 0 ? ctx->U : ctx->st64.lv[level - 1];
    launch_links_to_aos(l, ci.off, ci.V, ctx->staging, ctx->stream);
    MAG_TRY(ctx->check("mag_stout_level"));
    MAG_CUDA(cudaMemcpyAsync(host, ctx->staging, sizeof(double) * 72 * (size_t)ci.V, cudaMemcpyDeviceToHost,
                             ctx->stream));
    return ctx->sync("mag_stout_level");
}

int mag_integrate(mag_ctx* ctx) {
    if (!ctx) return MAG_ERR_ARG;
    MAG_TRY(ctx->ensure_tuned());
    MAG_TRY(ctx->integrate());
    return ctx->sync("mag_integrate");
}

int mag_trajectory(mag_ctx* ctx, int refresh, mag_traj_result* results) {
    if (!ctx) return MAG_ERR_ARG;
    MAG_TRY(ctx->ensure_tuned());
    MAG_TRY(ctx->trajectory_body(refresh != 0));
    std::vector<TrajRecord> r(ctx->nchain);
    MAG_CUDA(cudaMemcpyAsync(r.data(), ctx->rec, sizeof(TrajRecord) * ctx->nchain, cudaMemcpyDeviceToHost,
                             ctx->stream));
    MAG_TRY(ctx->sync("mag_trajectory"));
    ctx->host_traj++;
    bool finite = true;
    for (int c = 0; c < ctx->nchain; c++) {
        if (results) mag_ctx::to_result(r[c], &results[c]);
        finite = finite && std::isfinite(r[c].delta_h);
    }
    if (!finite) return fail(MAG_ERR_NAN, "non-finite Delta H");
    return MAG_OK;
}

namespace {

// n_sweeps demon sweeps of the chains `chains` (all of one context), each on an AoS copy of its
// links: one CTA per chain and sweep launch.  Outputs per listed chain j: demon_energy[(j *
// n_sweeps + i) * 4 + k], reunit[j * n_sweeps + i], accepted[j], rejected[j] (any may be NULL).
int demon_sweeps(mag_ctx* ctx, const std::vector<int>& chains, const std::vector<unsigned long long>& seeds,
                 int n_sweeps, double e_max, int update_links, double* demon_energy, int64_t* accepted,
                 int64_t* rejected, double* reunit) {
    const int nj = (int)chains.size();
    if (!ctx->d_demon_tables) {
        std::unique_ptr<DemonTables> tabs(new DemonTables);
        if (!build_demon_tables(tabs.get())) return fail(MAG_ERR_ARG, "demon path window overflow");
        MAG_TRY(ctx->alloc((void**)&ctx->d_demon_tables, sizeof(DemonTables)));
        MAG_TRY(ctx->alloc((void**)&ctx->d_demon, sizeof(DemonState) * ctx->nchain));
        MAG_TRY(ctx->alloc((void**)&ctx->d_demon_jobs, sizeof(DemonJob) * ctx->nchain));
        MAG_CUDA(cudaMemcpyAsync(ctx->d_demon_tables, tabs.get(), sizeof(DemonTables), cudaMemcpyHostToDevice,
                                 ctx->stream));
        MAG_TRY(ctx->sync("demon tables"));
    }
    // one chain: its AoS copy in the staging buffer; several: the ensemble-wide AoS buffer
    double* aos = ctx->staging;
    if (nj > 1) {
        if (!ctx->demon_aos) MAG_TRY(ctx->alloc((void**)&ctx->demon_aos, sizeof(double) * 72 * (size_t)ctx->vpad));
        aos = ctx->demon_aos;
    }
    std::vector<DemonJob> jobs(nj);
    for (int j = 0; j < nj; j++) {
        const ChainInfo& ci = ctx->hc[chains[j]];
        jobs[j].ci = ci;
        jobs[j].aos_off = nj > 1 ? 36LL * ci.off : 0;
        jobs[j].seed = seeds[j];
    }
    // the reference sweeps a copy of the field (field-demon.h:47-49) and starts the demons at 0 (:44);
    // the copy is kept in the reject backup (which only a trajectory in progress uses) and swept as
    // AoS links, then converted back for the reunitarisation after each sweep
    const std::vector<DemonState> zero(nj, DemonState{{0.0, 0.0, 0.0, 0.0}, 0, 0});
    MAG_CUDA(cudaMemcpyAsync(ctx->d_demon_jobs, jobs.data(), sizeof(DemonJob) * nj, cudaMemcpyHostToDevice,
                             ctx->stream));
    MAG_CUDA(cudaMemcpyAsync(ctx->d_demon, zero.data(), sizeof(DemonState) * nj, cudaMemcpyHostToDevice,
                             ctx->stream));
    LinkPlanes<double> work = ctx->Ubak;
    launch_link_copy(ctx->geom, ctx->U, work, ctx->stream);
    MAG_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    std::vector<DemonState> st(nj);
    std::vector<unsigned long long> bits(ctx->nchain);
    for (int i = 0; i < n_sweeps; i++) {
        for (int j = 0; j < nj; j++) {
            const ChainInfo& ci = ctx->hc[chains[j]];
            launch_links_to_aos(work, ci.off, ci.V, aos + 2 * jobs[j].aos_off, ctx->stream);
        }
        launch_demon_sweeps(ctx->d_demon_jobs, nj, aos, ctx->d_demon_tables, i, e_max, ctx->d_demon, ctx->stream);
        for (int j = 0; j < nj; j++) {
            const ChainInfo& ci = ctx->hc[chains[j]];
            launch_aos_to_links(aos + 2 * jobs[j].aos_off, ci.off, ci.V, work, ctx->vpad, ctx->stream);
        }
        // field-demon.h:111 reunitarizes the swept field after every sweep
        MAG_CUDA(cudaMemsetAsync(ctx->reunit, 0, sizeof(unsigned long long) * ctx->nchain, ctx->stream));
        launch_reunitarize(ctx->geom, work, LinkPlanes<float>{nullptr, 0}, ctx->reunit, ctx->stream);
        MAG_CUDA(cudaMemcpyAsync(st.data(), ctx->d_demon, sizeof(DemonState) * nj, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        MAG_CUDA(cudaMemcpyAsync(bits.data(), ctx->reunit, sizeof(unsigned long long) * ctx->nchain,
                                 cudaMemcpyDeviceToHost, ctx->stream));
        MAG_TRY(ctx->sync("mag_demon_microcanonical"));
        for (int j = 0; j < nj; j++) {
            if (demon_energy)
                for (int k = 0; k < 4; k++) demon_energy[((size_t)j * n_sweeps + i) * 4 + k] = st[j].E[k];
            if (reunit) {
                double d;
                memcpy(&d, &bits[chains[j]], sizeof(d));
                reunit[(size_t)j * n_sweeps + i] = d;
            }
        }
    }
    MAG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    MAG_TRY(ctx->sync("mag_demon_microcanonical"));
    float ms = 0.f;
    MAG_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_measure_ms = ms;
    for (int j = 0; j < nj; j++) {
        if (accepted) accepted[j] = n_sweeps ? st[j].accept : 0;
        if (rejected) rejected[j] = n_sweeps ? st[j].reject : 0;
    }
    if (update_links) {
        launch_link_copy(ctx->geom, work, ctx->U, ctx->stream);
        MAG_TRY(ctx->refresh_copy());
    }
    return ctx->sync("mag_demon_microcanonical");
}

}  // namespace

int mag_demon_microcanonical(mag_ctx* ctx, int chain, int n_sweeps, double e_max, uint64_t seed,
                             int update_links, double* demon_energy, int64_t* accepted, int64_t* rejected,
                             double* reunit) {
    if (!ctx || n_sweeps < 0 || !(e_max >= 0.0)) return fail(MAG_ERR_ARG, "mag_demon_microcanonical: bad argument");
    MAG_TRY(ctx->chain_ok(chain));
    return demon_sweeps(ctx, {chain}, {(unsigned long long)seed}, n_sweeps, e_max, update_links, demon_energy,
                        accepted, rejected, reunit);
}

int mag_demon_microcanonical_all(mag_ctx* ctx, int n_sweeps, double e_max, uint64_t seed, int update_links,
                                 double* demon_energy, int64_t* accepted, int64_t* rejected, double* reunit) {
    if (!ctx || n_sweeps < 0 || !(e_max >= 0.0))
        return fail(MAG_ERR_ARG, "mag_demon_microcanonical_all: bad argument");
    std::vector<int> chains(ctx->nchain);
    std::vector<unsigned long long> seeds(ctx->nchain);
    for (int c = 0; c < ctx->nchain; c++) {
        chains[c] = c;
        seeds[c] = (unsigned long long)seed + ctx->h_stream_index[c];
    }
    return demon_sweeps(ctx, chains, seeds, n_sweeps, e_max, update_links, demon_energy, accepted, rejected, reunit);
}

int mag_fg_trajectory(mag_ctx* ctx, int refresh_momenta, mag_traj_result* results) {
    return mag_trajectory(ctx, refresh_momenta, results);
}

int mag_batch_create(const mag_params* p, int n_chains, mag_ctx** out) {
    return mag_ensemble_create(p, n_chains, out);
}

int mag_batch_run(mag_ctx* ctx, int n_traj, mag_traj_result* results) { return mag_run(ctx, n_traj, results); }

int mag_run(mag_ctx* ctx, int n_traj, mag_traj_result* results) {
    if (!ctx || n_traj < 0) return MAG_ERR_ARG;
    MAG_TRY(ctx->build_graph());
    std::vector<TrajRecord> r;
    double total = 0.0;
    bool finite = true;
    for (int done = 0; done < n_traj;) {
        const int chunk = std::min(kHistCap, n_traj - done);
        const long long base = ctx->host_traj;
        MAG_CUDA(cudaMemcpyAsync(ctx->hist_base, &base, sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
        MAG_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
        for (int i = 0; i < chunk; i++) MAG_CUDA(cudaGraphLaunch(ctx->graph, ctx->stream));
        MAG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
        r.resize((size_t)chunk * ctx->nchain);
        MAG_CUDA(cudaMemcpyAsync(r.data(), ctx->hist, sizeof(TrajRecord) * r.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
        MAG_TRY(ctx->sync("mag_run"));
        float ms = 0.f;
        MAG_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        total += ms;
        for (size_t k = 0; k < r.size(); k++) {
            if (results) mag_ctx::to_result(r[k], &results[(size_t)done * ctx->nchain + k]);
            finite = finite && std::isfinite(r[k].delta_h);
        }
        ctx->host_traj += chunk;
        done += chunk;
    }
    ctx->last_run_ms = total;
    if (!finite) return fail(MAG_ERR_NAN, "non-finite Delta H");
    return MAG_OK;
}

int mag_set_stream_index(mag_ctx* ctx, const int64_t* index) {
    if (!ctx || !index) return fail(MAG_ERR_ARG, "mag_set_stream_index: null argument");
    std::vector<unsigned long long> v(ctx->nchain);
    for (int c = 0; c < ctx->nchain; c++) {
        if (index[c] < 0) return fail(MAG_ERR_ARG, "mag_set_stream_index: negative index");
        v[c] = (unsigned long long)index[c];
    }
    MAG_CUDA(cudaMemcpyAsync(ctx->d_stream_index, v.data(), sizeof(unsigned long long) * v.size(),
                             cudaMemcpyHostToDevice, ctx->stream));
    MAG_TRY(ctx->sync("mag_set_stream_index"));
    ctx->h_stream_index = v;
    return MAG_OK;
}

int mag_traj_counter(mag_ctx* ctx, int64_t* traj) {
    if (!ctx || !traj) return MAG_ERR_ARG;
    *traj = ctx->host_traj;
    return MAG_OK;
}

int mag_set_traj_counter(mag_ctx* ctx, int64_t traj) {
    if (!ctx || traj < 0) return MAG_ERR_ARG;
    const long long t = traj;
    MAG_CUDA(cudaMemcpyAsync(ctx->traj_counter, &t, sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    ctx->host_traj = traj;
    return ctx->sync("mag_set_traj_counter");
}

int mag_last_run_ms(mag_ctx* ctx, double* total_ms) {
    if (!ctx || !total_ms) return MAG_ERR_ARG;
    *total_ms = ctx->last_run_ms;
    return MAG_OK;
}

int mag_last_measure_ms(mag_ctx* ctx, double* ms) {
    if (!ctx || !ms) return MAG_ERR_ARG;
    *ms = ctx->last_measure_ms;
    return MAG_OK;
}

int mag_time_force(mag_ctx* ctx, int reps, double* ms) {
    if (!ctx || !ms || reps < 1) return MAG_ERR_ARG;
    auto once = [&]() {
        if (ctx->mixed) ctx->force_eval<float>(ctx->U32, ctx->F32, ctx->st32);
        else ctx->force_eval<double>(ctx->U, ctx->F, ctx->st64);
    };
    once();
    MAG_TRY(ctx->sync("mag_time_force warm-up"));
    MAG_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int i = 0; i < reps; i++) once();
    MAG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    MAG_TRY(ctx->sync("mag_time_force"));
    float t = 0.f;
    MAG_CUDA(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    *ms = t / reps;
    return MAG_OK;
}

}  // extern "C"
namespace {
// CRC segments: about two per resident thread of a 148-SM device, at least 256 bytes each
constexpr size_t kCrcThreads = 148 * 2048 * 2;
constexpr int kCrcGroup = 64;  // segment registers folded per thread on the device
size_t crc_seg(size_t bytes) {
    const size_t s = (bytes + kCrcThreads - 1) / kCrcThreads;
    return std::max<size_t>(256, (s + 15) / 16 * 16);
}
int nersc_buffers(mag_ctx* ctx);
int ensure_crc_tab(mag_ctx* ctx, size_t seg);
}  // namespace
namespace {
const char* const kFamNames[KF_COUNT] = {"force", "staple", "stout_forward", "stout_lambda", "stout_chain"};
// variant names: one thread per link at minimum blocks per SM 2..5 ("t1m2".."t1m5"); direction split with
// NS warps per 32-link tile at register cap R ("s<NS>r<R>")
const char* const kVariantNames[kNumVariants] = {"t1m2", "t1m3", "t1m4", "t1m5", "s3r168",
                                                  "s3r128", "s6r168", "s6r128", "s6r96"};
}  // namespace

extern "C" {

int mag_time_kernel(mag_ctx* ctx, const char* which, int reps, double* ms) {
    if (!ctx || !which || !ms || reps < 1) return MAG_ERR_ARG;
    const std::string w(which);
    const bool m = ctx->mixed;
    const int L = ctx->p.n_stout;
    auto& g = ctx->geom;
    cudaStream_t s = ctx->stream;
    int fam = -1;
    for (int f = 0; f < KF_COUNT; f++)
        if (w == kFamNames[f]) fam = f;
    if (fam >= KF_STOUT_FWD && L == 0) return fail(MAG_ERR_STATE, "mag_time_kernel: no stout levels in this context");
    MAG_TRY(ctx->ensure_tuned());
    // one full force evaluation first, so every intermediate buffer holds live data
    if (m) ctx->force_eval<float>(ctx->U32, ctx->F32, ctx->st32);
    else ctx->force_eval<double>(ctx->U, ctx->F, ctx->st64);
    if (fam >= 0) {
        const KernelFamily f = (KernelFamily)fam;
        if (m) return ctx->time_one<float>(f, ctx->var<float>(f), reps, ctx->st32, ctx->U32, ctx->F32, ctx->Uaux32, ms);
        return ctx->time_one<double>(f, ctx->var<double>(f), reps, ctx->st64, ctx->U, ctx->F, ctx->Uaux, ms);
    }
    std::function<void()> fn;
    if (w.rfind("nersc_", 0) == 0) {
        // NERSC payload kernels on chain 0's full (3x3) payload, made from the current links
        MAG_TRY(nersc_buffers(ctx));
        const ChainInfo& c0 = ctx->hc[0];
        const size_t bytes = (size_t)c0.V * 4 * 9 * 16;
        launch_links_to_payload(ctx->U, 0, c0.off, c0.V, ctx->staging, s);
        if (w == "nersc_swap") {
            fn = [&]() { launch_swap64_sum32(ctx->staging, bytes, true, ctx->d_csum, s); };
        } else if (w == "nersc_crc") {
            const size_t seg = crc_seg(bytes);
            MAG_TRY(ensure_crc_tab(ctx, seg));
            fn = [&, seg]() {
                launch_crc32_segments(ctx->staging, bytes, seg, ctx->d_crc, s);
                launch_crc32_fold(ctx->d_crc, bytes / seg, kCrcGroup, ctx->d_crc_tab, ctx->d_crc2, s);
            };
        } else if (w == "nersc_to_links") {  // rewrites the same links bit for bit
            fn = [&]() { launch_payload_to_links(ctx->staging, 0, c0.off, c0.V, ctx->U, s); };
        } else if (w == "nersc_from_links") {
            fn = [&]() { launch_links_to_payload(ctx->U, 0, c0.off, c0.V, ctx->staging, s); };
        } else if (w == "nersc_plaq") {  // the plaquette and link-trace sums of the import check
            fn = [&]() {
                launch_action_sums<double>(g, ctx->U, false, ctx->partial, ctx->sums, SLOT_SCRATCH, SLOT_SCRATCH, s);
                launch_link_trace_sum(g, ctx->U, ctx->partial, ctx->sums, SLOT_SCRATCH2, s);
            };
        } else {
            return fail(MAG_ERR_ARG, "mag_time_kernel: unknown kernel '" + w + "'");
        }
    } else if (w == "evolve") {
        fn = [&]() {
            launch_evolve<double, double>(g, ctx->U, ctx->Ubak, ctx->P, 1e-3,
                                          m ? ctx->Uaux32 : LinkPlanes<float>{nullptr, 0}, s);
        };
    } else if (w == "kick") {
        fn = [&]() {
            if (m) launch_kick<float>(g, ctx->P, ctx->F32, 0.0, s);
            else launch_kick<double>(g, ctx->P, ctx->F, 0.0, s);
        };
    } else if (w == "action") {
        fn = [&]() {
            launch_action_sums<double>(g, ctx->U, true, ctx->partial, ctx->sums, SLOT_SCRATCH, SLOT_SCRATCH, s);
        };
    } else {
        return fail(MAG_ERR_ARG, "mag_time_kernel: unknown kernel '" + w + "'");
    }
    fn();
    MAG_TRY(ctx->sync("mag_time_kernel warm-up"));
    MAG_CUDA(cudaEventRecord(ctx->ev0, s));
    for (int i = 0; i < reps; i++) fn();
    MAG_CUDA(cudaEventRecord(ctx->ev1, s));
    MAG_TRY(ctx->sync("mag_time_kernel"));
    float t = 0.f;
    MAG_CUDA(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    *ms = t / reps;
    return MAG_OK;
}


int mag_autotune(mag_ctx* ctx, int reps, char* report, size_t len) {
    if (!ctx || reps < 1) return MAG_ERR_ARG;
    MAG_TRY(ctx->autotune(reps));
    if (report && len) {
        std::string r = "{";
        for (int f = 0; f < KF_COUNT; f++) {
            if (f) r += ", ";
            r += std::string("\"") + kFamNames[f] + "\": {";
            for (int pi = 0; pi < 2; pi++) {
                r += std::string(pi ? ", " : "") + "\"" + (pi ? "fp32" : "fp64") + "\": [\"" +
                     kVariantNames[ctx->tune[f][pi]] + "\", {";
                bool first = true;
                for (int v = 0; v < kNumVariants; v++) {
                    if (ctx->tune_ms[f][pi][v] <= 0.0) continue;
                    char b[64];
                    std::snprintf(b, sizeof b, "%s\"%s\": %.5f", first ? "" : ", ", kVariantNames[v],
                                  ctx->tune_ms[f][pi][v]);
                    r += b;
                    first = false;
                }
                r += "}]";
            }
            r += "}";
        }
        // block traversal order of the link kernels (0: raster, T: T x T tiles of (x2, x3) rows)
        char b[160];
        std::snprintf(b, sizeof b, ", \"block_order\": [%d, {\"raster\": %.5f, \"tile2\": %.5f, \"tile4\": %.5f}]",
                      ctx->geom.tile, ctx->tile_time_ms[0], ctx->tile_time_ms[1], ctx->tile_time_ms[2]);
        r += b;
        r += "}";
        if (r.size() + 1 > len) return fail(MAG_ERR_ARG, "mag_autotune: report buffer too small");
        std::snprintf(report, len, "%s", r.c_str());
    }
    return MAG_OK;
}

int mag_set_kernel_variant(mag_ctx* ctx, const char* family, int precision, const char* variant) {
    if (!ctx || !family || !variant || precision < 0 || precision > 1) return MAG_ERR_ARG;
    int f = -1, v = -1;
    for (int k = 0; k < KF_COUNT; k++)
        if (!std::strcmp(family, kFamNames[k])) f = k;
    for (int k = 0; k < kNumVariants; k++)
        if (!std::strcmp(variant, kVariantNames[k])) v = k;
    if (f < 0) return fail(MAG_ERR_ARG, std::string("mag_set_kernel_variant: unknown family '") + family + "'");
    if (v < 0 || v >= mag_ctx::variants_of((KernelFamily)f))
        return fail(MAG_ERR_ARG, std::string("mag_set_kernel_variant: no variant '") + variant + "' for " + family);
    MAG_TRY(ctx->ensure_tuned());
    ctx->tune[f][precision] = v;
    if (ctx->graph) {  // the captured trajectory holds the previous choice
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
    return MAG_OK;
}

int mag_graph_kernel_count(mag_ctx* ctx, int* kernels) {
    if (!ctx || !kernels) return MAG_ERR_ARG;
    MAG_TRY(ctx->build_graph());
    *kernels = ctx->graph_kernels;
    return MAG_OK;
}

int mag_expiq(const double* q, int64_t n, double* out) {
    const double* in[1] = {q};
    return matrix_op("mag_expiq", in, 1, n, out, [&](const double* dq, const double*, const double*, double* o) {
        launch_expiq(dq, (long)n, o, 0);
    });
}

int mag_dexpiq(const double* q, const double* dq, int64_t n, double* out) {
    const double* in[2] = {q, dq};
    return matrix_op("mag_dexpiq", in, 2, n, out, [&](const double* d0, const double* d1, const double*, double* o) {
        launch_dexpiq(d0, d1, (long)n, o, 0);
    });
}

int mag_compute_lambda(const double* q, const double* sigma, const double* u, int64_t n, double* lambda) {
    const double* in[3] = {q, sigma, u};
    return matrix_op("mag_compute_lambda", in, 3, n, lambda,
                     [&](const double* dq, const double* ds, const double* du, double* o) {
                         launch_compute_lambda(dq, ds, du, (long)n, o, 0);
                     });
}

int mag_probe_fma_peak(int precision, double* tflops) {
    if (!tflops || precision < 0 || precision > 2) return MAG_ERR_ARG;
    int dev = 0, sms = 0;
    MAG_CUDA(cudaGetDevice(&dev));
    MAG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int nblocks = sms * 8, iters = precision == 0 ? 2048 : 8192;
    void* out = nullptr;
    MAG_CUDA(cudaMalloc(&out, (size_t)nblocks * 256 * 8));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int rep = 0; rep < 6; rep++) {
        cudaEventRecord(a, 0);
        if (precision == 0) launch_fma_probe<double>((double*)out, nblocks, iters, 0);
        else if (precision == 1) launch_fma_probe<float>((float*)out, nblocks, iters, 0);
        else launch_ffma2_probe(out, nblocks, iters, 0);
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    MAG_CUDA(cudaGetLastError());
    // two flops per FMA; a packed f32x2 FMA is two FMAs
    *tflops = (precision == 2 ? 4.0 : 2.0) * 8.0 * iters * (double)nblocks * 256 / (best * 1e-3) / 1e12;
    return MAG_OK;
}

// closed paths summed over sites (or coarse sites) of one chain, double-double
static int run_paths(mag_ctx* ctx, int chain, const std::vector<int>& dirs, int npath, int plen, int coarse_mag,
                     double* sum) {
    MAG_TRY(ctx->ensure_meas(1, 1, false));
    if ((int)dirs.size() > ctx->max_path_ints) return fail(MAG_ERR_ARG, "path too long");
    MAG_CUDA(cudaMemcpyAsync(ctx->d_paths, dirs.data(), sizeof(int) * dirs.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
    launch_wilson_general(ctx->geom, ctx->U, ctx->d_paths, npath, plen, coarse_mag, ctx->wl_partial, ctx->wl_out,
                          ctx->stream);
    MAG_TRY(ctx->check("paths"));
    std::vector<dd2> out(ctx->nchain);
    MAG_CUDA(cudaMemcpyAsync(out.data(), ctx->wl_out, sizeof(dd2) * ctx->nchain, cudaMemcpyDeviceToHost,
                             ctx->stream));
    MAG_TRY(ctx->sync("paths"));
    *sum = out[chain].hi + out[chain].lo;
    return MAG_OK;
}

int mag_wilson_loop(mag_ctx* ctx, int chain, const int r[3], int T, double* out) {
    if (!ctx || !r || !out || T < 1) return fail(MAG_ERR_ARG, "mag_wilson_loop: bad arguments");
    MAG_TRY(ctx->chain_ok(chain));
    for (int i = 0; i < 3; i++)
        if (r[i] < 0) return fail(MAG_ERR_ARG, "mag_wilson_loop: negative r");
    // permutations of the sorted r (field-wloop.h:66-71) and their paths (:32-50)
    std::vector<int> rl(r, r + 3);
    std::sort(rl.begin(), rl.end());
    std::vector<std::vector<int>> paths;
    do {
        std::vector<int> d;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < rl[i]; j++) d.push_back(i);
        for (int j = 0; j < T; j++) d.push_back(3);
        for (int i = 2; i >= 0; i--)
            for (int j = 0; j < rl[i]; j++) d.push_back(i + 4);
        for (int j = 0; j < T; j++) d.push_back(7);
        paths.push_back(d);
    } while (std::next_permutation(rl.begin(), rl.end()));
    const int plen = (int)paths[0].size();
    std::vector<int> flat;
    for (auto& p : paths) flat.insert(flat.end(), p.begin(), p.end());
    double s = 0.0;
    MAG_TRY(run_paths(ctx, chain, flat, (int)paths.size(), plen, 0, &s));
    *out = s / ((double)paths.size() * ctx->hc[chain].V);
    return MAG_OK;
}

int mag_wilson_loops(mag_ctx* ctx, int chain, int Rmax, int Tmax, double* out) {
    if (!ctx || !out || Rmax < 1 || Tmax < 1 || Rmax > 64 || Tmax > 64)
        return fail(MAG_ERR_ARG, "mag_wilson_loops: bad arguments");
    MAG_TRY(ctx->chain_ok(chain));
    MAG_TRY(ctx->ensure_meas(Rmax, Tmax, true));
    const long vp = ctx->vpad;
    LinkPlanes<double> lines{ctx->wl_lines, vp};
    LinkPlanes<double> tl{ctx->wl_lines + (size_t)Rmax * 9 * vp, vp};
    LinkPlanes<double> tl2{ctx->wl_lines + (size_t)(Rmax + 1) * 9 * vp, vp};
    MAG_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    launch_wilson_planar(ctx->geom, ctx->U, Rmax, Tmax, lines, tl, tl2, ctx->wl_partial, ctx->wl_out, ctx->stream);
    MAG_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    MAG_TRY(ctx->check("mag_wilson_loops"));
    const size_t n = (size_t)3 * Tmax * ctx->nchain * Rmax;
    std::vector<dd2> h(n);
    MAG_CUDA(cudaMemcpyAsync(h.data(), ctx->wl_out, sizeof(dd2) * n, cudaMemcpyDeviceToHost, ctx->stream));
    MAG_TRY(ctx->sync("mag_wilson_loops"));
    float wl_ms = 0.f;
    MAG_CUDA(cudaEventElapsedTime(&wl_ms, ctx->ev0, ctx->ev1));
    ctx->last_measure_ms = wl_ms;
    const double norm = 3.0 * ctx->hc[chain].V;  // perm.size() * V (field-wloop.h:98)
    for (int R = 1; R <= Rmax; R++)
        for (int T = 1; T <= Tmax; T++) {
            hdd acc{0.0, 0.0};
            for (int i = 0; i < 3; i++) {
                const dd2 v = h[((size_t)(i * Tmax + T - 1) * ctx->nchain + chain) * Rmax + R - 1];
                acc = h_add(acc, hdd{v.hi, v.lo});
            }
            out[(R - 1) * Tmax + (T - 1)] = (acc.hi + acc.lo) / norm;
        }
    return MAG_OK;
}

int mag_constrained_plaquette(mag_ctx* ctx, int chain, double* out) {
    if (!ctx || !out) return MAG_ERR_ARG;
    MAG_TRY(ctx->chain_ok(chain));
    const int m = ctx->hc[chain].mag;
    if (m < 1) return fail(MAG_ERR_STATE, "mag_constrained_plaquette: chain has no constraint (mag = 0)");
    // mag x mag loops in the six planes mu > nu from every coarse site (field-matrix.h:418-436)
    std::vector<int> flat;
    int npath = 0;
    for (int mu = 0; mu < 4; mu++)
        for (int nu = 0; nu < mu; nu++) {
            for (int i = 0; i < m; i++) flat.push_back(mu);
            for (int i = 0; i < m; i++) flat.push_back(nu);
            for (int i = 0; i < m; i++) flat.push_back(mu + 4);
            for (int i = 0; i < m; i++) flat.push_back(nu + 4);
            npath++;
        }
    double s = 0.0;
    MAG_TRY(run_paths(ctx, chain, flat, npath, 4 * m, m, &s));
    long coarse = 1;
    for (int d = 0; d < 4; d++) coarse *= ctx->hc[chain].L[d] / m;
    *out = s / (3.0 * (double)(coarse * npath));
    return MAG_OK;
}

}  // extern "C"

// ------------------------------------------------------------- NERSC I/O
namespace {

constexpr size_t kIoChunk = 8u << 20;      // pinned chunk of the file <-> device copies

// reader / writer threads of the file <-> device pipeline (two pinned slots each)
int io_threads() {
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(2u, std::min(8u, hc / 2));
}

void fill_info(mag_nersc_info* info, const nersc::Header& h, int two_row) {
    memset(info, 0, sizeof(*info));
    for (int d = 0; d < 4; d++) info->dims[d] = h.dims[d];
    info->two_row = two_row;
    info->payload_offset = h.payload_offset;
    info->checksum_header = h.checksum;
    info->crc32_header = h.crc32;
    info->plaquette_header = h.plaquette;
    info->link_trace_header = h.link_trace;
}

struct FileCloser {
    FILE* f;
    ~FileCloser() {
        if (f) fclose(f);
    }
};

int nersc_buffers(mag_ctx* ctx) {
    std::string err;
    int r = ctx->pin.ensure(2 * io_threads(), kIoChunk, err);
    if (r != MAG_OK) return fail(r, err);
    if (!ctx->d_crc) {
        MAG_TRY(ctx->alloc((void**)&ctx->d_crc, sizeof(uint32_t) * (kCrcThreads + 1)));
        MAG_TRY(ctx->alloc((void**)&ctx->d_crc2, sizeof(uint32_t) * (kCrcThreads / kCrcGroup + 1)));
        MAG_TRY(ctx->alloc((void**)&ctx->d_crc_tab, sizeof(uint32_t) * 4 * 256));
        MAG_TRY(ctx->alloc((void**)&ctx->d_csum, sizeof(unsigned int)));
    }
    return MAG_OK;
}

// avg_plaquette (field-matrix.h:387-389) and avg_real_trace (:391-405) of one chain
int plaq_and_trace(mag_ctx* ctx, int chain, double* plaq, double* trace) {
    launch_action_sums<double>(ctx->geom, ctx->U, false, ctx->partial, ctx->sums, SLOT_SCRATCH, SLOT_SCRATCH,
                               ctx->stream);
    launch_link_trace_sum(ctx->geom, ctx->U, ctx->partial, ctx->sums, SLOT_SCRATCH2, ctx->stream);
    MAG_TRY(ctx->check("NERSC plaquette"));
    std::vector<dd2> s;
    MAG_TRY(ctx->read_sums(s));
    const double V = (double)ctx->hc[chain].V;
    const dd2 pl = s[chain * NUM_SLOTS + SLOT_SCRATCH], tr = s[chain * NUM_SLOTS + SLOT_SCRATCH2];
    *plaq = (pl.hi + pl.lo) / (18.0 * V);
    *trace = (tr.hi + tr.lo) / (12.0 * V);
    return MAG_OK;
}

// CRC-32 of the host-order payload in staging and its 32-bit word sum; to_be
// leaves the payload big-endian (export), else it is converted to host order
// first (import)
int ensure_crc_tab(mag_ctx* ctx, size_t seg) {
    if (ctx->crc_tab_seg == seg) return MAG_OK;
    uint32_t tab[4][256];
    nersc::crc32_shift_tables(seg, tab);
    MAG_CUDA(cudaMemcpyAsync(ctx->d_crc_tab, tab, sizeof(tab), cudaMemcpyHostToDevice, ctx->stream));
    MAG_TRY(ctx->sync("crc tables"));
    ctx->crc_tab_seg = seg;
    return MAG_OK;
}

int payload_digest(mag_ctx* ctx, size_t bytes, bool import, uint32_t* crc, uint32_t* csum) {
    const size_t seg = crc_seg(bytes);
    const size_t nfull = bytes / seg, tail = bytes - nfull * seg;
    const size_t ngroups = (nfull + kCrcGroup - 1) / kCrcGroup;
    MAG_TRY(ensure_crc_tab(ctx, seg));
    MAG_CUDA(cudaMemsetAsync(ctx->d_csum, 0, sizeof(unsigned int), ctx->stream));
    if (import) launch_swap64_sum32(ctx->staging, bytes, true, ctx->d_csum, ctx->stream);
    launch_crc32_segments(ctx->staging, bytes, seg, ctx->d_crc, ctx->stream);
    launch_crc32_fold(ctx->d_crc, nfull, kCrcGroup, ctx->d_crc_tab, ctx->d_crc2, ctx->stream);
    if (!import) launch_swap64_sum32(ctx->staging, bytes, false, ctx->d_csum, ctx->stream);
    MAG_TRY(ctx->check("NERSC payload digest"));
    std::vector<uint32_t> z2(ngroups + 1);
    unsigned int sum = 0;
    if (ngroups)
        MAG_CUDA(cudaMemcpyAsync(z2.data(), ctx->d_crc2, sizeof(uint32_t) * ngroups, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    if (tail)
        MAG_CUDA(cudaMemcpyAsync(&z2[ngroups], ctx->d_crc + nfull, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    MAG_CUDA(cudaMemcpyAsync(&sum, ctx->d_csum, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    MAG_TRY(ctx->sync("NERSC payload digest"));
    // zlib: register started at ~0, result complemented; groups of kCrcGroup segments, the last group shorter
    uint32_t r = 0xFFFFFFFFu;
    if (ngroups) {
        const size_t last = (nfull - (ngroups - 1) * kCrcGroup) * seg;
        r = nersc::crc32_fold(r, z2.data(), ngroups, kCrcGroup * seg, last);
    }
    if (tail) r = nersc::crc32_fold(r, &z2[ngroups], 1, tail, tail);
    *crc = ~r;
    *csum = sum;
    return MAG_OK;
}

}  // namespace

extern "C" {

int mag_nersc_read_header(const char* path, mag_nersc_info* info) {
    if (!path || !info) return fail(MAG_ERR_ARG, "mag_nersc_read_header: null argument");
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(MAG_ERR_IO, std::string("cannot open ") + path);
    nersc::Header h;
    std::string err;
    int two_row = 0;
    int r = nersc::read_header(fc.f, h, err);
    if (r == MAG_OK) r = nersc::datatype_rows(h.datatype, two_row, err);
    if (r != MAG_OK) return fail(r, std::string("import_config_nersc: ") + err);
    fill_info(info, h, two_row);
    return MAG_OK;
}

int mag_gauge_load_nersc(mag_ctx* ctx, int chain, const char* path, mag_nersc_info* info) {
    if (!ctx || !path) return fail(MAG_ERR_ARG, "mag_gauge_load_nersc: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(MAG_ERR_IO, std::string("cannot open ") + path);
    nersc::Header h;
    std::string err;
    int two_row = 0;
    int r = nersc::read_header(fc.f, h, err);
    if (r == MAG_OK) r = nersc::datatype_rows(h.datatype, two_row, err);
    if (r != MAG_OK) return fail(r, std::string("import_config_nersc: ") + err);
    for (int d = 0; d < 4; d++)
        if (h.dims[d] != ci.L[d])
            return fail(MAG_ERR_FORMAT, "import_config_nersc: WRONG Lattice Size (file " + std::to_string(h.dims[0]) +
                                            "x" + std::to_string(h.dims[1]) + "x" + std::to_string(h.dims[2]) + "x" +
                                            std::to_string(h.dims[3]) + ")");
    MAG_TRY(nersc_buffers(ctx));
    const size_t bytes = (size_t)ci.V * 4 * (two_row ? 6 : 9) * 16;
    r = nersc::file_to_device(fileno(fc.f), h.payload_offset, ctx->staging, bytes, ctx->pin, io_threads(),
                              ctx->stream, err);
    if (r != MAG_OK) return fail(r, "import_config_nersc: " + err);
    uint32_t crc = 0, csum = 0;
    MAG_TRY(payload_digest(ctx, bytes, true, &crc, &csum));
    if (info) {
        fill_info(info, h, two_row);
        info->checksum = csum;
        info->crc32 = crc;
    }
    // field-matrix.h:673-676 / :695-699: the links are left untouched on a checksum mismatch
    if (csum != h.checksum) {
        char b[128];
        snprintf(b, sizeof(b), "import_config_nersc: WRONG Checksum: %x(labeled) vs %x(computed)", h.checksum, csum);
        return fail(MAG_ERR_CHECKSUM, b);
    }
    launch_payload_to_links(ctx->staging, two_row, ci.off, ci.V, ctx->U, ctx->stream);
    MAG_TRY(ctx->refresh_copy());
    double plaq = 0.0, trace = 0.0;
    MAG_TRY(plaq_and_trace(ctx, chain, &plaq, &trace));
    if (info) {
        info->plaquette = plaq;
        info->link_trace = trace;
    }
    // field-matrix.h:708-711
    if (std::fabs(plaq - h.plaquette) > 1e-4) {
        char b[160];
        snprintf(b, sizeof(b), "import_config_nersc: Plaquette: %.8f(labeled) vs %.8f(computed)", h.plaquette, plaq);
        return fail(MAG_ERR_PLAQUETTE, b);
    }
    return MAG_OK;
}

int mag_gauge_save_nersc(mag_ctx* ctx, int chain, const char* path, int two_row, double beta,
                         int sequence_number, const char* ensemble_label, mag_nersc_info* info) {
    if (!ctx || !path) return fail(MAG_ERR_ARG, "mag_gauge_save_nersc: null argument");
    MAG_TRY(ctx->chain_ok(chain));
    const ChainInfo& ci = ctx->hc[chain];
    MAG_TRY(nersc_buffers(ctx));
    double plaq = 0.0, trace = 0.0;
    MAG_TRY(plaq_and_trace(ctx, chain, &plaq, &trace));
    const size_t bytes = (size_t)ci.V * 4 * (two_row ? 6 : 9) * 16;
    launch_links_to_payload(ctx->U, two_row ? 1 : 0, ci.off, ci.V, ctx->staging, ctx->stream);
    uint32_t crc = 0, csum = 0;
    MAG_TRY(payload_digest(ctx, bytes, false, &crc, &csum));
    const std::string hdr = nersc::format_header(ci.L, two_row ? 1 : 0, crc, csum, trace, plaq, ensemble_label,
                                                 sequence_number, beta, (long long)time(nullptr));
    const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return fail(MAG_ERR_IO, std::string("cannot create ") + path);
    std::string err;
    int r = MAG_OK;
    if (pwrite(fd, hdr.data(), hdr.size(), 0) != (ssize_t)hdr.size()) {
        r = MAG_ERR_IO;
        err = "header write failed";
    }
    if (r == MAG_OK)
        r = nersc::device_to_file(ctx->staging, bytes, fd, (long long)hdr.size(), ctx->pin, io_threads(),
                                  ctx->stream, err);
    if (close(fd) != 0 && r == MAG_OK) {
        r = MAG_ERR_IO;
        err = "close failed";
    }
    if (r != MAG_OK) return fail(r, "export_config_nersc: " + err);
    if (info) {
        memset(info, 0, sizeof(*info));
        for (int d = 0; d < 4; d++) info->dims[d] = ci.L[d];
        info->two_row = two_row ? 1 : 0;
        info->payload_offset = (int64_t)hdr.size();
        info->checksum_header = info->checksum = csum;
        info->crc32_header = info->crc32 = crc;
        info->plaquette_header = info->plaquette = plaq;
        info->link_trace_header = info->link_trace = trace;
    }
    return MAG_OK;
}

int mag_crc32_host(const void* data, size_t n, size_t seg, uint32_t* crc) {
    if ((!data && n) || !crc || seg == 0 || seg % 16) return fail(MAG_ERR_ARG, "mag_crc32_host: bad argument");
    const uint8_t* p = static_cast<const uint8_t*>(data);
    const size_t nseg = (n + seg - 1) / seg;
    std::vector<uint32_t> z(nseg);
    for (size_t i = 0; i < nseg; i++) z[i] = nersc::crc32_register(p + i * seg, std::min(seg, n - i * seg));
    *crc = nersc::crc32_chain(z.data(), nseg, seg, n);
    return MAG_OK;
}

}  // extern "C"

// ------------------------------------------------------------ domain decomposition
// A lattice split along x3 into n shards (fetch_expanded_chart's halo exchange,
// field-hmc.h:544-558, with the expansion of run_chmc, field-hmc.h:777-781).
// Each shard is an ordinary context over its slab of Lloc = L3 / n time slices
// plus h halo slices on either side; every kernel runs on the whole extended
// slab (the halo's results are discarded), and the context's hook refreshes the
// halo slices from the neighbouring shards' interiors wherever a later kernel
// reads across the boundary.  Sums (kinetic energy, plaquette and rectangle
// sums) run over interior sites and are added over the shards before the
// accept step (the reference's MPI_Allreduce, field-hmc.h:628, and MPI_Bcast of
// the decision, :823), so every shard takes the same decision.
//
// In one process the shards are driven by one host thread each (the hook
// meets the other threads at a barrier; no kernel ever waits for another):
// a halo is filled by device-to-device copies on the receiving shard's stream
// after it has waited on the sending shard's event.
struct mag_dd {
    int n = 0, h = 0, device = 0;
    std::vector<mag_ctx*> shards;
    std::vector<cudaEvent_t> ready, copied;
    std::vector<void*> base;
    std::vector<std::vector<dd2>> host_sums;
    std::vector<unsigned long long> host_reunit;
    std::vector<double> staging;  // one shard's extended AoS field
    // reusable barrier for the shard threads
    std::mutex mu;
    std::condition_variable cv;
    int arrived = 0;
    long generation = 0;
    void barrier() {
        std::unique_lock<std::mutex> lk(mu);
        const long gen = generation;
        if (++arrived == n) {
            arrived = 0;
            generation++;
            cv.notify_all();
        } else {
            cv.wait(lk, [&] { return generation != gen; });
        }
    }
    ~mag_dd() {
        for (auto e : ready) cudaEventDestroy(e);
        for (auto e : copied) cudaEventDestroy(e);
        for (auto c : shards) delete c;
    }
    // run fn(rank) for every shard, one host thread each; first non-OK status wins
    int run(const std::function<int(int)>& fn) {
        std::vector<int> rc(n, MAG_OK);
        std::vector<std::thread> th;
        for (int r = 0; r < n; r++)
            th.emplace_back([&, r] {
                cudaSetDevice(device);
                rc[r] = fn(r);
            });
        for (auto& t : th) t.join();
        for (int r = 0; r < n; r++)
            if (rc[r] != MAG_OK) return rc[r];
        return MAG_OK;
    }
    long slab_sites() const { return (long)shards[0]->hc[0].L[0] * shards[0]->hc[0].L[1] * shards[0]->hc[0].L[2]; }
};

namespace {

struct DdHook : HaloHook {
    mag_dd* d;
    explicit DdHook(mag_dd* dd) : d(dd) {}
    int exchange(mag_ctx* c, void* base, size_t unit) override {
        const int s = c->shard_rank, n = d->n, lo = (s + n - 1) % n, hi = (s + 1) % n;
        const ChainInfo& ci = c->hc[0];
        d->base[s] = base;
        cudaError_t e = cudaEventRecord(d->ready[s], c->stream);
        d->barrier();
        const size_t S3 = (size_t)d->slab_sites(), slab = (size_t)d->h * S3 * unit, plane = unit * (size_t)c->vpad;
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, d->ready[lo], 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, d->ready[hi], 0);
        for (int mu = 0; mu < 4 && e == cudaSuccess; mu++) {
            char* dst = static_cast<char*>(base) + mu * plane;
            const char* src_lo = static_cast<const char*>(d->base[lo]) + mu * plane;
            const char* src_hi = static_cast<const char*>(d->base[hi]) + mu * plane;
            // low halo <- the lower shard's top interior slices; high halo <- the upper shard's bottom ones
            e = cudaMemcpyAsync(dst, src_lo + (size_t)(ci.hi3 - d->h) * S3 * unit, slab, cudaMemcpyDeviceToDevice,
                                c->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(dst + (size_t)ci.hi3 * S3 * unit, src_hi + (size_t)ci.lo3 * S3 * unit, slab,
                                    cudaMemcpyDeviceToDevice, c->stream);
        }
        if (e == cudaSuccess) e = cudaEventRecord(d->copied[s], c->stream);
        d->barrier();
        // the neighbours' copies out of this shard finish before this shard writes the field again
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, d->copied[lo], 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, d->copied[hi], 0);
        if (e != cudaSuccess) return fail(MAG_ERR_CUDA, std::string("halo exchange: ") + cudaGetErrorString(e));
        return MAG_OK;
    }
    int reduce(mag_ctx* c, const int* slots, int nslots, bool reunit) override {
        const int s = c->shard_rank;
        std::vector<dd2>& mine = d->host_sums[s];
        cudaError_t e = cudaMemcpyAsync(mine.data(), c->sums, sizeof(dd2) * NUM_SLOTS, cudaMemcpyDeviceToHost,
                                        c->stream);
        if (e == cudaSuccess && reunit)
            e = cudaMemcpyAsync(&d->host_reunit[s], c->reunit, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        d->barrier();
        // every shard adds the shards' sums in the same order, so all hold the same totals
        std::vector<dd2> tot = mine;
        for (int k = 0; k < nslots; k++) {
            hdd acc{0.0, 0.0};
            for (int r = 0; r < d->n; r++) acc = h_add(acc, hdd{d->host_sums[r][slots[k]].hi, d->host_sums[r][slots[k]].lo});
            tot[slots[k]] = dd2{acc.hi, acc.lo};
        }
        unsigned long long rmax = 0;
        if (reunit)
            for (int r = 0; r < d->n; r++) rmax = std::max(rmax, d->host_reunit[r]);  // non-negative doubles
        d->barrier();
        // on the shard's stream (a plain cudaMemcpy from pageable memory may return before the
        // copy lands, and the shard's non-blocking stream would not wait for it), then synchronised
        // because the host values live in this frame
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c->sums, tot.data(), sizeof(dd2) * NUM_SLOTS, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess && reunit)
            e = cudaMemcpyAsync(c->reunit, &rmax, sizeof(rmax), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return fail(MAG_ERR_CUDA, std::string("halo reduce: ") + cudaGetErrorString(e));
        return MAG_OK;
    }
};

// lattice AoS field (x0 fastest, 72 doubles per site) <-> one shard's extended slab
void dd_slab(const mag_dd* d, int r, const double* lattice, double* shard, bool to_shard, bool interior_only) {
    const ChainInfo& ci = d->shards[r]->hc[0];
    const size_t per = 72 * (size_t)d->slab_sites();
    for (int x3 = 0; x3 < ci.L[3]; x3++) {
        if (interior_only && (x3 < ci.lo3 || x3 >= ci.hi3)) continue;
        int g3 = (x3 + ci.org3) % ci.L3g;
        if (g3 < 0) g3 += ci.L3g;
        if (to_shard) std::memcpy(shard + x3 * per, lattice + g3 * per, per * sizeof(double));
        else std::memcpy(const_cast<double*>(lattice) + g3 * per, shard + x3 * per, per * sizeof(double));
    }
}

}  // namespace

// argument checks shared by mag_dd_create and mag_shard_create
int shard_args(const mag_params* p, int nshards, int halo, const char* who) {
    const int L3 = p->dims[3];
    if (nshards < 1 || L3 % nshards) return fail(MAG_ERR_ARG, std::string(who) + ": dims[3] must divide into the shards");
    const int loc = L3 / nshards;
    if (halo < 2 || halo > loc) return fail(MAG_ERR_ARG, std::string(who) + ": halo depth must be in [2, dims[3] / nshards]");
    if (p->mag > 0 && loc % p->mag)
        return fail(MAG_ERR_ARG, std::string(who) + ": a shard's dims[3] / nshards must be a multiple of mag");
    if (((long)p->dims[0] * p->dims[1] * p->dims[2]) % MAG_TILE)
        return fail(MAG_ERR_ARG, std::string(who) + ": dims[0] dims[1] dims[2] must be a multiple of 32");
    return MAG_OK;
}

// One slab per process (or thread): the caller moves the halos itself through
// a callback (MPI, NCCL, gloo), as qlat's fetch_expanded_chart does through MPI.
struct CallbackHook : HaloHook {
    mag_halo_fn fn;
    void* user;
    CallbackHook(mag_halo_fn f, void* u) : fn(f), user(u) {}
    int exchange(mag_ctx* c, void* base, size_t unit) override {
        const ChainInfo& ci = c->hc[0];
        const size_t S3 = (size_t)ci.L[0] * ci.L[1] * ci.L[2];
        mag_halo_op op{};
        op.kind = MAG_HALO_EXCHANGE;
        op.base = base;
        op.nplanes = 4;
        op.plane_bytes = unit * (size_t)c->vpad;
        op.slab_bytes = (size_t)c->shard_h * S3 * unit;
        op.send_lo = (size_t)ci.lo3 * S3 * unit;
        op.send_hi = (size_t)(ci.hi3 - c->shard_h) * S3 * unit;
        op.recv_lo = 0;
        op.recv_hi = (size_t)ci.hi3 * S3 * unit;
        op.stream = c->stream;
        op.rank = c->shard_rank;
        op.nshards = c->shard_n;
        const int rc = fn(user, &op);
        if (rc != 0) return fail(MAG_ERR_STATE, "halo exchange callback returned " + std::to_string(rc));
        return MAG_OK;
    }
    int reduce(mag_ctx* c, const int* slots, int nslots, bool reunit) override {
        std::vector<dd2> h(NUM_SLOTS);
        unsigned long long r = 0;
        MAG_CUDA(cudaMemcpyAsync(h.data(), c->sums, sizeof(dd2) * NUM_SLOTS, cudaMemcpyDeviceToHost, c->stream));
        if (reunit) MAG_CUDA(cudaMemcpyAsync(&r, c->reunit, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
        MAG_TRY(c->sync("halo reduce"));
        std::vector<double> v(2 * (size_t)nslots);
        for (int k = 0; k < nslots; k++) {
            v[2 * k] = h[slots[k]].hi;
            v[2 * k + 1] = h[slots[k]].lo;
        }
        double rmax = 0.0;
        std::memcpy(&rmax, &r, sizeof(r));
        mag_halo_op op{};
        op.kind = MAG_HALO_SUM;
        op.sums = v.data();
        op.nsums = 2 * nslots;
        op.maxval = reunit ? &rmax : nullptr;
        op.stream = c->stream;
        op.rank = c->shard_rank;
        op.nshards = c->shard_n;
        const int rc = fn(user, &op);
        if (rc != 0) return fail(MAG_ERR_STATE, "halo reduce callback returned " + std::to_string(rc));
        for (int k = 0; k < nslots; k++) {
            // the slabs' (hi, lo) pairs were added componentwise: renormalise
            const double hi = v[2 * k], lo = v[2 * k + 1];
            const double sum = hi + lo;
            h[slots[k]] = dd2{sum, lo - (sum - hi)};
        }
        std::memcpy(&r, &rmax, sizeof(r));
        MAG_CUDA(cudaMemcpyAsync(c->sums, h.data(), sizeof(dd2) * NUM_SLOTS, cudaMemcpyHostToDevice, c->stream));
        if (reunit) MAG_CUDA(cudaMemcpyAsync(c->reunit, &r, sizeof(r), cudaMemcpyHostToDevice, c->stream));
        return c->sync("halo reduce");
    }
};

extern "C" {

int mag_dd_create(const mag_params* p, int nshards, int halo, mag_dd** out) {
    if (!p || !out) return fail(MAG_ERR_ARG, "mag_dd_create: null argument");
    *out = nullptr;
    MAG_TRY(shard_args(p, nshards, halo, "mag_dd_create"));
    mag_dd* d = new mag_dd();
    d->n = nshards;
    d->h = halo;
    cudaGetDevice(&d->device);
    for (int r = 0; r < nshards; r++) {
        mag_ctx* c = new mag_ctx();
        const int spec[3] = {nshards, r, halo};
        const int rc = c->init(p, 1, spec);
        if (rc != MAG_OK) {
            delete c;
            delete d;
            return rc;
        }
        d->shards.push_back(c);
    }
    d->ready.resize(nshards);
    d->copied.resize(nshards);
    for (int r = 0; r < nshards; r++) {
        if (cudaEventCreateWithFlags(&d->ready[r], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&d->copied[r], cudaEventDisableTiming) != cudaSuccess) {
            delete d;
            return fail(MAG_ERR_CUDA, "mag_dd_create: event creation failed");
        }
    }
    d->base.assign(nshards, nullptr);
    d->host_sums.assign(nshards, std::vector<dd2>(NUM_SLOTS));
    d->host_reunit.assign(nshards, 0);
    d->staging.resize(72 * (size_t)d->shards[0]->hc[0].V);
    // launch shapes are tuned once on shard 0 (without exchanges) and shared
    mag_ctx* c0 = d->shards[0];
    int rc = c0->ensure_tuned();
    for (int r = 1; r < nshards && rc == MAG_OK; r++) {
        std::memcpy(d->shards[r]->tune, c0->tune, sizeof(c0->tune));
        d->shards[r]->tuned = true;
    }
    if (rc != MAG_OK) {
        delete d;
        return rc;
    }
    for (auto c : d->shards) c->halo = new DdHook(d);
    *out = d;
    return MAG_OK;
}

int mag_dd_destroy(mag_dd* d) {
    if (!d) return MAG_ERR_ARG;
    for (auto c : d->shards) {
        delete c->halo;
        c->halo = nullptr;
    }
    delete d;
    return MAG_OK;
}

int mag_dd_gauge_set(mag_dd* d, const double* host) {
    if (!d || !host) return fail(MAG_ERR_ARG, "mag_dd_gauge_set: null argument");
    for (int r = 0; r < d->n; r++) {
        dd_slab(d, r, host, d->staging.data(), true, false);
        MAG_TRY(mag_gauge_set(d->shards[r], 0, d->staging.data()));
    }
    return MAG_OK;
}

int mag_dd_gauge_get(mag_dd* d, double* host) {
    if (!d || !host) return fail(MAG_ERR_ARG, "mag_dd_gauge_get: null argument");
    for (int r = 0; r < d->n; r++) {
        MAG_TRY(mag_gauge_get(d->shards[r], 0, d->staging.data()));
        dd_slab(d, r, host, d->staging.data(), false, true);
    }
    return MAG_OK;
}

int mag_dd_momentum_set(mag_dd* d, const double* host) {
    if (!d || !host) return fail(MAG_ERR_ARG, "mag_dd_momentum_set: null argument");
    for (int r = 0; r < d->n; r++) {
        dd_slab(d, r, host, d->staging.data(), true, false);
        MAG_TRY(mag_momentum_set(d->shards[r], 0, d->staging.data()));
    }
    return MAG_OK;
}

int mag_dd_momentum_get(mag_dd* d, double* host) {
    if (!d || !host) return fail(MAG_ERR_ARG, "mag_dd_momentum_get: null argument");
    for (int r = 0; r < d->n; r++) {
        MAG_TRY(mag_momentum_get(d->shards[r], 0, d->staging.data()));
        dd_slab(d, r, host, d->staging.data(), false, true);
    }
    return MAG_OK;
}

int mag_dd_hot_start(mag_dd* d, uint64_t seed) {
    if (!d) return MAG_ERR_ARG;
    for (auto c : d->shards) MAG_TRY(mag_gauge_hot_start(c, seed));
    return MAG_OK;
}

int mag_dd_uniforms_set(mag_dd* d, const double* u) {
    if (!d) return MAG_ERR_ARG;
    for (auto c : d->shards) MAG_TRY(mag_uniforms_set(c, u));
    return MAG_OK;
}

int mag_dd_gauge_force(mag_dd* d, double* host) {
    if (!d || !host) return fail(MAG_ERR_ARG, "mag_dd_gauge_force: null argument");
    MAG_TRY(d->run([&](int r) {
        mag_ctx* c = d->shards[r];
        c->halo_rc = MAG_OK;
        if (c->mixed) c->force_eval<float>(c->U32, c->F32, c->st32);
        else c->force_eval<double>(c->U, c->F, c->st64);
        if (c->halo_rc != MAG_OK) return c->halo_rc;
        return c->sync("mag_dd_gauge_force");
    }));
    for (int r = 0; r < d->n; r++) {
        mag_ctx* c = d->shards[r];
        const ChainInfo& ci = c->hc[0];
        if (c->mixed) launch_alg_to_aos<float>(c->F32, ci.off, ci.V, c->staging, c->stream);
        else launch_alg_to_aos<double>(c->F, ci.off, ci.V, c->staging, c->stream);
        MAG_CUDA(cudaMemcpyAsync(d->staging.data(), c->staging, sizeof(double) * 72 * (size_t)ci.V,
                                 cudaMemcpyDeviceToHost, c->stream));
        MAG_TRY(c->sync("mag_dd_gauge_force"));
        dd_slab(d, r, host, d->staging.data(), false, true);
    }
    return MAG_OK;
}

int mag_dd_trajectory(mag_dd* d, int refresh, mag_traj_result* result) {
    if (!d) return MAG_ERR_ARG;
    std::vector<TrajRecord> rec(d->n);
    MAG_TRY(d->run([&](int r) {
        mag_ctx* c = d->shards[r];
        c->halo_rc = MAG_OK;
        int rc = c->trajectory_body(refresh != 0);
        if (rc != MAG_OK) return rc;
        if (cudaMemcpyAsync(&rec[r], c->rec, sizeof(TrajRecord), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
            return fail(MAG_ERR_CUDA, "mag_dd_trajectory: record copy");
        rc = c->sync("mag_dd_trajectory");
        if (rc == MAG_OK) c->host_traj++;
        return rc;
    }));
    for (int r = 1; r < d->n; r++)
        if (rec[r].accept != rec[0].accept || rec[r].delta_h != rec[0].delta_h)
            return fail(MAG_ERR_STATE, "mag_dd_trajectory: shards disagree on the accept step");
    if (result) mag_ctx::to_result(rec[0], result);
    if (!std::isfinite(rec[0].delta_h)) return fail(MAG_ERR_NAN, "mag_dd_trajectory: non-finite Delta H");
    return MAG_OK;
}

int mag_dd_shard(mag_dd* d, int rank, mag_ctx** ctx) {
    if (!d || !ctx || rank < 0 || rank >= d->n) return MAG_ERR_ARG;
    *ctx = d->shards[rank];
    return MAG_OK;
}

int mag_shard_create(const mag_params* p, int nshards, int rank, int halo, mag_ctx** out) {
    if (!p || !out) return fail(MAG_ERR_ARG, "mag_shard_create: null argument");
    *out = nullptr;
    MAG_TRY(shard_args(p, nshards, halo, "mag_shard_create"));
    if (rank < 0 || rank >= nshards) return fail(MAG_ERR_ARG, "mag_shard_create: rank out of range");
    mag_ctx* c = new mag_ctx();
    const int spec[3] = {nshards, rank, halo};
    const int rc = c->init(p, 1, spec);
    if (rc != MAG_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return MAG_OK;
}

int mag_set_halo_fn(mag_ctx* ctx, mag_halo_fn fn, void* user) {
    if (!ctx || !fn) return fail(MAG_ERR_ARG, "mag_set_halo_fn: null argument");
    if (ctx->shard_h == 0) return fail(MAG_ERR_STATE, "mag_set_halo_fn: not a shard context (mag_shard_create)");
    MAG_TRY(ctx->ensure_tuned());  // tuned before the hook: the tuner's force evaluations exchange nothing
    delete ctx->halo;
    ctx->halo = new CallbackHook(fn, user);
    if (ctx->graph) {
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
    return MAG_OK;
}

}  // extern "C"


// ------------------------------------------------------------ two-level coupling
// run_hmc_multi (field-multi.h:758-900): a fine lattice and a coarse lattice of
// half the extent in every direction, coupled through the stout-smeared blocked
// links of the fine field (kernels_multi.cu).  H = K_fine + K_coarse +
// S_gauge(fine) + S_eta; both fields move together in one force-gradient
// integration (force_gradient_integrator_multi, field-multi.h:685-756), unconstrained.
// The reference reads rho and eta_sqr from globals outside its tree; here they
// are arguments.  FP64 throughout; host-supplied momenta and uniform.
struct mag_multi {
    mag_ctx* f = nullptr;  // fine lattice (mag = 0, no stout levels of its own)
    mag_ctx* c = nullptr;  // coarse lattice
    double rho = 0.1, eta_sqr = 1.0;
    AlgPlanes<double> lam{nullptr, 0};
    LinkPlanes<double> zp{nullptr, 0};
    dd2* partial = nullptr;
    dd2* energy = nullptr;
    ~mag_multi() {
        delete f;
        delete c;
    }
    const ChainInfo& cf() const { return f->hc[0]; }
    const ChainInfo& cc() const { return c->hc[0]; }
    cudaStream_t s() const { return f->stream; }

    void forces(LinkPlanes<double> uf, LinkPlanes<double> uc) {
        f->force_eval<double>(uf, f->F, f->st64);  // thin gauge force of the fine field
        launch_multi_coarse(cf(), cc(), uf, uc, rho, eta_sqr, c->F, lam, zp, nullptr, nullptr, s());
        launch_multi_fine(cf(), cc(), uf, lam, zp, rho, eta_sqr, f->F, s());
    }
    void drift(double eps) {
        launch_evolve<double, double>(f->geom, f->U, f->U, f->P, eps, LinkPlanes<float>{nullptr, 0}, s());
        launch_evolve<double, double>(c->geom, c->U, c->U, c->P, eps, LinkPlanes<float>{nullptr, 0}, s());
    }
    void fg_kick(double dt, double gamma) {
        forces(f->U, c->U);
        launch_evolve<double, double>(f->geom, f->U, f->Uaux, f->F, gamma, LinkPlanes<float>{nullptr, 0}, s());
        launch_evolve<double, double>(c->geom, c->U, c->Uaux, c->F, gamma, LinkPlanes<float>{nullptr, 0}, s());
        forces(f->Uaux, c->Uaux);
        launch_kick<double>(f->geom, f->P, f->F, 0.5 * dt, s());
        launch_kick<double>(c->geom, c->P, c->F, 0.5 * dt, s());
    }
    int integrate(double dev[2]) {
        const mag_params& p = f->p;
        const double dt = p.tau / p.n_steps;
        const double alpha = (3. - std::sqrt(3.)) * dt / 6.;
        const double beta = dt / std::sqrt(3.);
        const double gamma = (2. - std::sqrt(3.)) * dt * dt / 12.;
        drift(alpha);
        for (int i = 0; i < p.n_steps; i++) {
            fg_kick(dt, gamma);
            drift(beta);
            fg_kick(dt, gamma);
            drift(i < p.n_steps - 1 ? 2. * alpha : alpha);
        }
        MAG_CUDA(cudaMemsetAsync(f->reunit, 0, sizeof(unsigned long long), s()));
        MAG_CUDA(cudaMemsetAsync(c->reunit, 0, sizeof(unsigned long long), s()));
        launch_reunitarize(f->geom, f->U, LinkPlanes<float>{nullptr, 0}, f->reunit, s());
        launch_reunitarize(c->geom, c->U, LinkPlanes<float>{nullptr, 0}, c->reunit, s());
        unsigned long long r[2];
        MAG_CUDA(cudaMemcpyAsync(&r[0], f->reunit, sizeof(r[0]), cudaMemcpyDeviceToHost, s()));
        MAG_CUDA(cudaMemcpyAsync(&r[1], c->reunit, sizeof(r[1]), cudaMemcpyDeviceToHost, s()));
        MAG_TRY(f->sync("multi integrate"));
        std::memcpy(dev, r, sizeof(r));
        return MAG_OK;
    }
    // {kinetic of both levels, fine gauge action, coupling energy} as double-double
    int hamiltonian(hdd parts[3]) {
        launch_kinetic_sum(f->geom, f->P, f->partial, f->sums, SLOT_KIN_OLD, s());
        launch_kinetic_sum(c->geom, c->P, c->partial, c->sums, SLOT_KIN_OLD, s());
        launch_action_sums<double>(f->geom, f->U, f->iwasaki, f->partial, f->sums, SLOT_PLAQ_OLD, SLOT_RECT_OLD, s());
        launch_multi_coarse(cf(), cc(), f->U, c->U, rho, eta_sqr, AlgPlanes<double>{nullptr, 0},
                            AlgPlanes<double>{nullptr, 0}, LinkPlanes<double>{nullptr, 0}, partial, energy, s());
        std::vector<dd2> sf(NUM_SLOTS), sc(NUM_SLOTS);
        dd2 e;
        MAG_CUDA(cudaMemcpyAsync(sf.data(), f->sums, sizeof(dd2) * NUM_SLOTS, cudaMemcpyDeviceToHost, s()));
        MAG_CUDA(cudaMemcpyAsync(sc.data(), c->sums, sizeof(dd2) * NUM_SLOTS, cudaMemcpyDeviceToHost, s()));
        MAG_CUDA(cudaMemcpyAsync(&e, energy, sizeof(dd2), cudaMemcpyDeviceToHost, s()));
        MAG_TRY(f->sync("multi hamiltonian"));
        parts[0] = h_add(hdd{sf[SLOT_KIN_OLD].hi, sf[SLOT_KIN_OLD].lo}, hdd{sc[SLOT_KIN_OLD].hi, sc[SLOT_KIN_OLD].lo});
        parts[1] = f->action_value(0, sf[SLOT_PLAQ_OLD], sf[SLOT_RECT_OLD]);
        parts[2] = h_mul(h_neg(hdd{e.hi, e.lo}), 1.0 / eta_sqr);  // -1/eta^2 sum ReTr(C^dag e^{iQ} V)
        return MAG_OK;
    }
};

extern "C" {

int mag_multi_create(const mag_params* fine, double rho, double eta_sqr, mag_multi** out) {
    if (!fine || !out) return fail(MAG_ERR_ARG, "mag_multi_create: null argument");
    *out = nullptr;
    for (int d = 0; d < 4; d++)
        if (fine->dims[d] < 4 || fine->dims[d] % 2)
            return fail(MAG_ERR_ARG, "mag_multi_create: fine extents must be even and >= 4");
    if (!(eta_sqr > 0.0)) return fail(MAG_ERR_ARG, "mag_multi_create: eta_sqr must be positive");
    mag_params pf = *fine;
    pf.mag = 0;
    pf.n_stout = 0;
    pf.precision = MAG_PREC_FP64;
    pf.integrator = MAG_INT_FORCE_GRADIENT;
    mag_params pc = pf;
    for (int d = 0; d < 4; d++) pc.dims[d] = fine->dims[d] / 2;
    mag_multi* m = new mag_multi();
    m->rho = rho;
    m->eta_sqr = eta_sqr;
    m->f = new mag_ctx();
    m->c = new mag_ctx();
    int r = m->f->init(&pf, 1);
    if (r == MAG_OK) r = m->c->init(&pc, 1);
    if (r == MAG_OK) r = m->c->alloc_alg(m->lam);
    if (r == MAG_OK) r = m->c->alloc_links(m->zp);
    const long nb = 4 * ((m->c->hc[0].V + 127) / 128);
    if (r == MAG_OK) r = m->c->alloc((void**)&m->partial, sizeof(dd2) * nb);
    if (r == MAG_OK) r = m->c->alloc((void**)&m->energy, sizeof(dd2));
    if (r == MAG_OK) r = m->f->ensure_tuned();
    if (r != MAG_OK) {
        delete m;
        return r;
    }
    *out = m;
    return MAG_OK;
}

int mag_multi_destroy(mag_multi* m) {
    if (!m) return MAG_ERR_ARG;
    delete m;
    return MAG_OK;
}

int mag_multi_gauge_set(mag_multi* m, const double* fine, const double* coarse) {
    if (!m || !fine || !coarse) return fail(MAG_ERR_ARG, "mag_multi_gauge_set: null argument");
    MAG_TRY(mag_gauge_set(m->f, 0, fine));
    return mag_gauge_set(m->c, 0, coarse);
}

int mag_multi_gauge_get(mag_multi* m, double* fine, double* coarse) {
    if (!m || !fine || !coarse) return fail(MAG_ERR_ARG, "mag_multi_gauge_get: null argument");
    MAG_TRY(mag_gauge_get(m->f, 0, fine));
    return mag_gauge_get(m->c, 0, coarse);
}

int mag_multi_momentum_set(mag_multi* m, const double* fine, const double* coarse) {
    if (!m || !fine || !coarse) return fail(MAG_ERR_ARG, "mag_multi_momentum_set: null argument");
    MAG_TRY(mag_momentum_set(m->f, 0, fine));
    return mag_momentum_set(m->c, 0, coarse);
}

int mag_multi_forces(mag_multi* m, double* fine_force, double* coarse_force) {
    if (!m || !fine_force || !coarse_force) return fail(MAG_ERR_ARG, "mag_multi_forces: null argument");
    m->forces(m->f->U, m->c->U);
    const ChainInfo &a = m->cf(), &b = m->cc();
    launch_alg_to_aos<double>(m->f->F, a.off, a.V, m->f->staging, m->s());
    MAG_CUDA(cudaMemcpyAsync(fine_force, m->f->staging, sizeof(double) * 72 * (size_t)a.V, cudaMemcpyDeviceToHost,
                             m->s()));
    launch_alg_to_aos<double>(m->c->F, b.off, b.V, m->c->staging, m->s());
    MAG_CUDA(cudaMemcpyAsync(coarse_force, m->c->staging, sizeof(double) * 72 * (size_t)b.V,
                             cudaMemcpyDeviceToHost, m->s()));
    return m->f->sync("mag_multi_forces");
}

int mag_multi_hamiltonian(mag_multi* m, double out[4]) {
    if (!m || !out) return MAG_ERR_ARG;
    hdd parts[3];
    MAG_TRY(m->hamiltonian(parts));
    const hdd h = h_add(h_add(parts[0], parts[1]), parts[2]);
    out[0] = h.hi + h.lo;
    for (int k = 0; k < 3; k++) out[k + 1] = parts[k].hi + parts[k].lo;
    return MAG_OK;
}

int mag_multi_trajectory(mag_multi* m, int traj_index, double uniform, double out[6]) {
    if (!m || !out) return MAG_ERR_ARG;
    launch_link_copy(m->f->geom, m->f->U, m->f->Ubak, m->s());
    launch_link_copy(m->c->geom, m->c->U, m->c->Ubak, m->s());
    hdd a[3], b[3];
    MAG_TRY(m->hamiltonian(a));
    double dev[2];
    MAG_TRY(m->integrate(dev));
    MAG_TRY(m->hamiltonian(b));
    // Delta H from the compensated parts
    hdd dh{0.0, 0.0};
    for (int k = 0; k < 3; k++) dh = h_add(dh, h_add(b[k], h_neg(a[k])));
    const double d = dh.hi + dh.lo;
    bool acc = uniform < std::exp(-d);
    if (traj_index < m->f->p.n_forced_accept) acc = true;
    if (!acc) {
        launch_link_copy(m->f->geom, m->f->Ubak, m->f->U, m->s());
        launch_link_copy(m->c->geom, m->c->Ubak, m->c->U, m->s());
        MAG_TRY(m->f->sync("mag_multi_trajectory"));
    }
    const hdd h0 = h_add(h_add(a[0], a[1]), a[2]), h1 = h_add(h_add(b[0], b[1]), b[2]);
    out[0] = h0.hi + h0.lo;
    out[1] = h1.hi + h1.lo;
    out[2] = d;
    out[3] = acc ? 1.0 : 0.0;
    out[4] = dev[0];
    out[5] = dev[1];
    if (!std::isfinite(d)) return fail(MAG_ERR_NAN, "mag_multi_trajectory: non-finite Delta H");
    return MAG_OK;
}

}  // extern "C"
