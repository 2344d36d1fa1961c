/*
 * mag_oracle.h -- C API of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle restates, in plain C++17 + OpenMP, the arithmetic of mag's
 * constrained hybrid Monte Carlo path (field-hmc.h, field-matrix.h, the stout
 * math of field-multi.h, field-wloop.h and the trajectory-level demon of
 * field-demon.h).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it, and only as a checker: the product never links it.
 *
 * PARITY UNPINNED: the reference ships no golden vectors and cannot be built
 * here (it needs CPS, Qlattice, QMP and MPI).  The restatement is checked
 * against invariants instead (unitarity, gauge invariance, finite-difference
 * derivatives, reversibility, dt^2 scaling, constraint invariance).
 *
 * Layout of every field argument: host AoS double[V][4][3][3][2], site index
 * x0 + L0*(x1 + L1*(x2 + L2*x3)) (x0 fastest, as qlat's index_from_coordinate).
 */
#ifndef MAG_ORACLE_H
#define MAG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mo_params {
    int dims[4];
    int mag;          /* 0: unconstrained; >=2 constrained segments (field-hmc.h:309) */
    int action;       /* 0 Wilson, 1 Iwasaki */
    double beta;
    double c1;        /* rectangle coefficient; c0 = 1 - 8 c1 */
    double rho;       /* stout parameter */
    int n_stout;      /* number of stout levels (0 = thin links) */
    double tau;       /* trajectory length */
    int n_steps;      /* integrator steps, dt = tau / n_steps */
    int integrator;   /* 0 force gradient (field-hmc.h:525), 1 leapfrog (:569) */
    int accept;       /* 0 Metropolis (field-hmc.h:818), 1 demon (field-demon.h:173) */
    double e_max;     /* demon window */
    int n_forced;     /* forced accepts at the start (field-hmc.h:826) */
} mo_params;

typedef struct mo_traj {
    double h_old, h_new, delta_h;
    double kin_old, kin_new, pot_old, pot_new;
    double plaq_old, plaq_new, rect_old, rect_new; /* raw sums of ReTr */
    double uniform;
    double demon[2];
    double reunit_maxdev;
    double avg_plaquette;
    int accept;
} mo_traj;

void mo_set_threads(int n);
int mo_get_threads(void);

/* Philox-4x32-10 block (Salmon et al., SC'11). */
void mo_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void mo_gen_hot(const int dims[4], uint64_t seed, double* U);
void mo_gen_momenta(const int dims[4], uint64_t seed, uint64_t traj, double* P);
double mo_gen_uniform(uint64_t seed, uint64_t traj);

/* single-matrix SU(3) helpers (18 doubles each) */
void mo_expiQ(const double* Q, double* out);
void mo_dexpiQ(const double* Q, const double* DQ, double* out);
void mo_compute_lambda(const double* Q, const double* SigmaP, const double* U, double* out);
void mo_unitarize(double* M);
void mo_ta(const double* M, double* out);

/* lattice-level operators */
void mo_plaq_rect(const int dims[4], const double* U, double out[2]);
double mo_avg_plaquette(const int dims[4], const double* U);
void mo_action(const mo_params* p, const double* U, double out[3]);
double mo_kinetic(const mo_params* p, const double* P);
void mo_staple_dagger(const mo_params* p, const double* U, double* V);
void mo_force(const mo_params* p, const double* U, double* F);
void mo_evolve_gauge(const mo_params* p, double* U, const double* P, double dt);
void mo_evolve_momentum(const int dims[4], double* P, const double* F, double dt, double m);
double mo_reunitarize(const int dims[4], double* U);
void mo_integrate(const mo_params* p, double* U, double* P, double* reunit_maxdev);
void mo_hamiltonian(const mo_params* p, const double* U, const double* P, double out[5]);
void mo_trajectory(const mo_params* p, int traj_index, double* U, const double* P,
                   double uniform, double demon[2], mo_traj* res);
void mo_run(const mo_params* p, uint64_t seed, int n_traj, double* U, mo_traj* res);
void mo_stout_forward(const mo_params* p, const double* U, double* levels);
double mo_wilson_loop(const int dims[4], const double* U, const int r[3], int T);
double mo_constrained_plaquette(const int dims[4], const double* U, int mag);
void mo_gauge_transform(const int dims[4], double* U, const double* G);

// field-demon.h:25-126 demon_microcanonical (per-link demons) on U in place
void mo_demon_sweeps(const int dims[4], double* U, uint64_t seed, int n_sweeps, double e_max, double* E_trace,
                     int64_t* accept, int64_t* reject, double* reunit);

/* two-level coupling (field-multi.h): coarse dims = dims / 2; rho, eta_sqr as parameters */
void mo_multi_forces(const mo_params* p, double rho, double eta_sqr, const double* Uf, const double* Uc, double* Ff,
                     double* Fc);
void mo_multi_hamiltonian(const mo_params* p, double rho, double eta_sqr, const double* Uf, const double* Pf,
                          const double* Uc, const double* Pc, double out[4]);
void mo_multi_trajectory(const mo_params* p, double rho, double eta_sqr, int traj_index, double* Uf,
                         const double* Pf, double* Uc, const double* Pc, double uniform, double out[6]);

#ifdef __cplusplus
}
#endif
#endif
