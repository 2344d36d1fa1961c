// mag_multi_api.cu -- the two-level coupling of field-multi.h (run_hmc_multi).
// The context is in ctx.h.
#include "ctx.h"

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

