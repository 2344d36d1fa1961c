// mag_dd.cu -- one lattice split into slabs along x3 with halo exchange: all
// slabs in one process (mag_dd_*), or one slab per process with the halos
// moved through a caller's callback (mag_shard_create, mag_set_halo_fn).
// The context is in ctx.h.
#include <exception>

#include "ctx.h"

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
    // reusable barrier for the shard threads; once broken (a shard thread could not be
    // started) every wait returns false at once, so the threads that did start finish
    std::mutex mu;
    std::condition_variable cv;
    int arrived = 0;
    long generation = 0;
    bool broken = false;
    bool barrier() {
        std::unique_lock<std::mutex> lk(mu);
        if (broken) return false;
        const long gen = generation;
        if (++arrived == n) {
            arrived = 0;
            generation++;
            cv.notify_all();
        } else {
            cv.wait(lk, [&] { return generation != gen || broken; });
        }
        return !broken;
    }
    void break_barrier() {
        std::lock_guard<std::mutex> lk(mu);
        broken = true;
        cv.notify_all();
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
        bool started = true;
        for (int r = 0; r < n; r++) {
            try {
                th.emplace_back([&, r] {
                    cudaSetDevice(device);
                    rc[r] = fn(r);
                });
            } catch (const std::exception&) {
                started = false;
                break_barrier();
                break;
            }
        }
        for (auto& t : th) t.join();
        {
            std::lock_guard<std::mutex> lk(mu);
            broken = false;
            arrived = 0;
        }
        if (!started) return fail(MAG_ERR_STATE, "domain decomposition: a shard thread could not be started");
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
        if (!d->barrier()) return fail(MAG_ERR_STATE, "halo exchange: the shard group is broken");
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
        if (!d->barrier()) return fail(MAG_ERR_STATE, "halo exchange: the shard group is broken");
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
        if (!d->barrier()) return fail(MAG_ERR_STATE, "halo reduce: the shard group is broken");
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
        if (!d->barrier()) return fail(MAG_ERR_STATE, "halo reduce: the shard group is broken");
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

}  // namespace

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


