// mag_api.cu -- C ABI of libmag_b200.so: contexts and ensembles, fields in and out,
// forces and MD pieces, trajectories and runs, measurements (Wilson loops, the
// constrained plaquette), per-matrix helpers, kernel timing and the tuner.  The
// context itself is in ctx.h.
#include "ctx.h"

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace magb {
// also lets the allocation-free entry point (noalloc.cu) report through mag_last_error()
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace magb

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
    if (!tflops || precision < 0 || precision > 3) return MAG_ERR_ARG;
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
        else launch_ffma2_probe(out, nblocks, iters, precision == 3, 0);
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
    *tflops = (precision >= 2 ? 4.0 : 2.0) * 8.0 * iters * (double)nblocks * 256 / (best * 1e-3) / 1e12;
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

