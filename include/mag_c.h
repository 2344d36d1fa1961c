/*
 * mag_c.h -- C ABI of libmag_b200.so, the B200 (sm_100a) implementation of
 * mag's constrained hybrid Monte Carlo path for SU(3) gauge fields.
 *
 * The reference (hummingtree/mag) exposes this path as free inline C++
 * functions over qlat::Field<cps::Matrix> (field-hmc.h, field-matrix.h,
 * field-multi.h, field-wloop.h, field-demon.h).  Each entry point below names
 * the reference function it replaces.  include/mag_field.hpp forwards the
 * reference names to these entry points for C++ drivers.
 *
 * Conventions
 *  - Every call returns int: MAG_OK (0) or a negative MAG_ERR_* code; no
 *    exception crosses the ABI (the reference asserts and aborts instead).
 *  - Host fields are AoS double[V][4][3][3][2] (site, mu, row, column, re/im),
 *    site index x0 + L0*(x1 + L1*(x2 + L2*x3)) as qlat's index_from_coordinate;
 *    momenta and forces use the same layout (Hermitian traceless matrices).
 *  - A context owns its device memory and one CUDA stream; it is not
 *    thread-safe (one host thread per context).  It holds one lattice or an
 *    ensemble of independent chains that advance in lockstep.
 *  - All randomness is Philox-4x32-10 keyed by (seed + chain index); a
 *    validation run may instead supply momenta and uniforms from the host.
 */
#ifndef MAG_C_H
#define MAG_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MAG_OK 0
#define MAG_ERR_ARG (-1)        /* invalid argument */
#define MAG_ERR_CUDA (-2)       /* CUDA runtime error (message: mag_last_error) */
#define MAG_ERR_NAN (-3)        /* NaN/Inf detected in a result */
#define MAG_ERR_STATE (-4)      /* call not valid in the current state */
#define MAG_ERR_NOMEM (-5)      /* device allocation failed */
#define MAG_ERR_IO (-6)         /* file could not be opened, read or written */
#define MAG_ERR_FORMAT (-7)     /* NERSC header: no END_HEADER, unknown DATATYPE, lattice size, short payload */
#define MAG_ERR_CHECKSUM (-8)   /* NERSC CHECKSUM differs from the payload */
#define MAG_ERR_PLAQUETTE (-9)  /* NERSC PLAQUETTE differs from the loaded links by more than 1e-4 */

enum { MAG_ACTION_WILSON = 0, MAG_ACTION_IWASAKI = 1 };           /* qlat::Gauge::type */
enum { MAG_PREC_FP64 = 0, MAG_PREC_MIXED = 1 };
enum { MAG_INT_FORCE_GRADIENT = 0, MAG_INT_LEAPFROG = 1 };
enum { MAG_ACCEPT_METROPOLIS = 0, MAG_ACCEPT_DEMON = 1 };

/* Arg_chmc (field-hmc.h:294-307) plus qlat::Gauge and the B200 run options. */
typedef struct mag_params {
    int dims[4];          /* lattice extents L0..L3 (each >= 2, divisible by mag) */
    int mag;              /* Arg_chmc::mag; 0 = unconstrained */
    int action;           /* MAG_ACTION_* */
    double beta;          /* Arg_chmc::beta */
    double c1;            /* Gauge::c1 (Iwasaki -0.331); c0 = 1 - 8 c1 */
    double rho;           /* stout parameter */
    int n_stout;          /* stout levels (0 = thin links) */
    double tau;           /* trajectory length; dt = tau / n_steps (Arg_chmc::dt) */
    int n_steps;          /* Arg_chmc::trajectory_length */
    int precision;        /* MAG_PREC_* */
    int integrator;       /* MAG_INT_* */
    int accept;           /* MAG_ACCEPT_* */
    double e_max;         /* demon window */
    int n_forced_accept;  /* Arg_chmc::num_forced_accept_step */
    uint64_t seed;        /* Philox key of chain 0 */
} mag_params;

/* One trajectory of one chain (the summary row of field-hmc.h:845-864). */
typedef struct mag_traj_result {
    double h_old, h_new, delta_h;
    double kinetic_old, kinetic_new, action_old, action_new;
    double plaq_sum_old, plaq_sum_new, rect_sum_old, rect_sum_new;
    double uniform;
    double demon[2];
    double reunit_maxdev;
    double avg_plaquette;
    int accept;
    int traj;
} mag_traj_result;

typedef struct mag_ctx mag_ctx;

/* -------------------------------------------------------------- lifecycle */
/* run_chmc's field set-up (field-hmc.h:775-784) for one lattice */
int mag_ctx_create(const mag_params* p, mag_ctx** out);
/* an ensemble of n independent chains (per-chain dims, mag, beta, c1, rho);
   precision, integrator, accept, n_stout, tau, n_steps and seed come from p[0] */
int mag_ensemble_create(const mag_params* p, int n_chains, mag_ctx** out);
int mag_ctx_destroy(mag_ctx* ctx);
const char* mag_last_error(void);
int mag_ctx_num_chains(const mag_ctx* ctx, int* n);
int mag_ctx_device_bytes(const mag_ctx* ctx, size_t* bytes);

/* ------------------------------------------------------------- field I/O */
/* copy a host configuration in / out (replaces gField = gFieldExt copies) */
int mag_gauge_set(mag_ctx* ctx, int chain, const double* host_aos);
int mag_gauge_get(mag_ctx* ctx, int chain, double* host_aos);
/* Haar-random hot start from Philox (seed + chain) / unit links */
int mag_gauge_hot_start(mag_ctx* ctx, uint64_t seed);
int mag_gauge_cold_start(mag_ctx* ctx);
/* momenta: init_momentum (field-hmc.h:675-693) from the host or from Philox */
int mag_momentum_set(mag_ctx* ctx, int chain, const double* host_aos);
int mag_momentum_get(mag_ctx* ctx, int chain, double* host_aos);
int mag_momentum_refresh(mag_ctx* ctx, uint64_t traj);
/* Metropolis uniforms for the next trajectory, one per chain (u_rand_gen, field-hmc.h:818);
   pass NULL to return to the Philox stream */
int mag_uniforms_set(mag_ctx* ctx, const double* u);

/* ------------------------------------------------------------- operators */
/* get_force (field-hmc.h:339-425) on the current links, smeared if n_stout > 0 */
int mag_gauge_force(mag_ctx* ctx, int chain, double* host_force_aos);
/* get_extended_staple_dagger (field-hmc.h:262-269) for every link of the
   (smeared) links */
int mag_staple(mag_ctx* ctx, int chain, double* host_staple_aos);
/* total_plaq / total_rectangular (field-matrix.h:299-385) of the smeared
   links and the gauge action (field-hmc.h:632-639) */
int mag_action(mag_ctx* ctx, int chain, double* plaq_sum, double* rect_sum, double* action);
/* avg_plaquette (field-matrix.h:387-389) of the thin links */
int mag_plaquette(mag_ctx* ctx, int chain, double* avg);
/* kinetic part of get_hamiltonian (field-hmc.h:596-629) */
int mag_kinetic(mag_ctx* ctx, int chain, double* kinetic);
/* get_hamiltonian (field-hmc.h:589-644): out = {H, kinetic, action} */
int mag_hamiltonian(mag_ctx* ctx, int chain, double out[3]);
/* evolve_gauge_field (field-hmc.h:442-482): U <- exp(i eps P) U with the constraint rules */
int mag_evolve_gauge(mag_ctx* ctx, double eps);
/* evolve_gauge_field driven by the momenta (MAG_SRC_MOMENTA, as mag_evolve_gauge) or by the
   force of the current links (MAG_SRC_FORCE: U <- exp(i eps F(U)) U, the force-gradient
   step's link update, field-hmc.h:497-503) */
enum { MAG_SRC_MOMENTA = 0, MAG_SRC_FORCE = 1 };
int mag_evolve_gauge_src(mag_ctx* ctx, double eps, int src);
/* evolve_momentum (field-hmc.h:427-440) with the force of the current links: P += eps F(U) */
int mag_evolve_momentum(mag_ctx* ctx, double eps);
/* reunitarize (field-matrix.h:83-100); maxdev[chain] = max |U' - U| */
int mag_reunitarize(mag_ctx* ctx, double* maxdev);
/* stout smearing forward of one chain: level k of the smeared links (k = 0 thin) */
int mag_stout_level(mag_ctx* ctx, int chain, int level, double* host_aos);
/* the same under the name of the stout entry points: mag_stout_forward = mag_stout_level;
   mag_stout_force = the force through the stout chain rule (mag_gauge_force of a context
   with n_stout >= 1; MAG_ERR_STATE without stout levels) */
int mag_stout_forward(mag_ctx* ctx, int chain, int level, double* host_aos);
int mag_stout_force(mag_ctx* ctx, int chain, double* host_force_aos);

/* ------------------------------------------------------------ integrator */
/* force_gradient_integrator (field-hmc.h:525-567) or leap_frog_integrator
   (field-hmc.h:569-587): one molecular-dynamics trajectory, no accept step */
int mag_integrate(mag_ctx* ctx);
/* one HMC trajectory of every chain (run_chmc loop body, field-hmc.h:806-843):
   H_old, integrate, reunitarize, H_new, Metropolis or demon accept, restore on
   reject.  refresh_momenta = 1 draws momenta from Philox for this trajectory;
   0 keeps the momenta set by mag_momentum_set.  results[chain] receives the
   record of each chain (may be NULL). */
int mag_trajectory(mag_ctx* ctx, int refresh_momenta, mag_traj_result* results);
/* n trajectories back to back with Philox momenta, the whole trajectory
   replayed as one CUDA graph; results[n * n_chains] in trajectory-major order */
int mag_run(mag_ctx* ctx, int n_traj, mag_traj_result* results);
/* the trajectory and ensemble entry points under their batch names:
   mag_fg_trajectory = mag_trajectory, mag_batch_create = mag_ensemble_create,
   mag_batch_run = mag_run */
int mag_fg_trajectory(mag_ctx* ctx, int refresh_momenta, mag_traj_result* results);
int mag_batch_create(const mag_params* p, int n_chains, mag_ctx** out);
int mag_batch_run(mag_ctx* ctx, int n_traj, mag_traj_result* results);
/* Philox stream of each chain: chain c's key is seed + index[c] for the hot start,
   the momenta and the Metropolis uniforms (default index[c] = c).  A job that splits
   one ensemble over several contexts (one per GPU) passes each chain's position in the
   whole ensemble, so every chain draws the numbers it would draw in one context. */
int mag_set_stream_index(mag_ctx* ctx, const int64_t* index);
/* number of trajectories done so far (the Philox trajectory counter) */
int mag_traj_counter(mag_ctx* ctx, int64_t* traj);
int mag_set_traj_counter(mag_ctx* ctx, int64_t traj);

/* ------------------------------------------------ single-matrix operators */
/* The reference's per-matrix helpers for n matrices at once.  Matrices are host arrays
   in the memory image of cps::Matrix: 9 complex doubles, row-major, re/im interleaved
   (double[n][3][3][2]).  Q must be Hermitian and traceless, as the reference assumes;
   its independent entries (diagonal 0, 1 and the upper triangle) are what is read.
   Both run on the current device with device buffers allocated for the call.
   expiQ (field-hmc.h:82-123): out[i] = exp(i Q[i]) by the Cayley-Hamilton closed form. */
int mag_expiq(const double* q, int64_t n, double* out);
/* DexpiQ (field-multi.h:90-178): out[i] = the derivative of exp(i Q) at Q[i] in the
   direction DQ[i] (any 3x3 matrix); zero where Q[i] = 0, as the reference returns. */
int mag_dexpiq(const double* q, const double* dq, int64_t n, double* out);
/* compute_Lambda (field-multi.h:180-269): lambda[i] = the Hermitian traceless part of
   Gamma(Q[i], SigmaP[i], U[i]), the stout chain rule's Lambda. */
int mag_compute_lambda(const double* q, const double* sigma, const double* u, int64_t n, double* lambda);

/* --------------------------------------------------- per-link demon sweep */
/* demon_microcanonical (field-demon.h:25-126) on one chain: n_sweeps sweeps over
   the links in site order (x0 fastest, mu inner) of a copy of the links, each link
   with its plaquette, rectangle, chair and twist staples (field-hmc.h:137-242,
   field-staple.h:27-149) and two hits of random_su3_from_su2(0.9) (field-matrix.h:36-65,
   drawn from Philox with this seed); a hit is accepted iff all four demons stay
   inside (-e_max, e_max).  The demons start at 0; after every sweep the field is
   reunitarized.  demon_energy[4 * i + k] = demon k after sweep i, reunit[i] = the
   reunitarisation's maximum deviation (either may be NULL); accepted / rejected count
   the hits.  update_links = 0 leaves the context's links as they were (the reference
   sweeps a copy); 1 keeps the swept field.  The sweep is sequential: one CTA walks
   the links, each link's 168 staple paths computed in parallel. */
int mag_demon_microcanonical(mag_ctx* ctx, int chain, int n_sweeps, double e_max, uint64_t seed,
                             int update_links, double* demon_energy, int64_t* accepted, int64_t* rejected,
                             double* reunit);
/* The same sweeps for every chain of an ensemble context at once, one CTA per chain
   (no reference counterpart: the reference sweeps one field).  Chain c draws with the
   Philox key seed + its stream index (the chain's index unless mag_set_stream_index
   changed it), so its result equals mag_demon_microcanonical(ctx, c, ..., seed + index).
   demon_energy[(c * n_sweeps + i) * 4 + k], reunit[c * n_sweeps + i], accepted[c],
   rejected[c] (any may be NULL). */
int mag_demon_microcanonical_all(mag_ctx* ctx, int n_sweeps, double e_max, uint64_t seed, int update_links,
                                 double* demon_energy, int64_t* accepted, int64_t* rejected, double* reunit);

/* ------------------------------------------------------------ measurement */
/* avg_wilson_loop (field-wloop.h:58-99) for a general spatial vector r and extent T */
int mag_wilson_loop(mag_ctx* ctx, int chain, const int r[3], int T, double* out);
/* planar loops R x T for R = 1..Rmax, T = 1..Tmax (r = (R,0,0) and its
   permutations); out[(R-1) * Tmax + (T-1)] */
int mag_wilson_loops(mag_ctx* ctx, int chain, int Rmax, int Tmax, double* out);
/* check_constrained_plaquette (field-matrix.h:407-443) */
int mag_constrained_plaquette(mag_ctx* ctx, int chain, double* out);

/* -------------------------------------------------------------- NERSC I/O */
/* Header fields and payload digests of a NERSC configuration file.  The
   payload is the lattice in site order x0 fastest, links mu = 0..3, each link
   rows 0-1 (DATATYPE 4D_SU3_GAUGE, two_row = 1) or the full matrix
   (4D_SU3_GAUGE_3x3), as big-endian IEEE-754 doubles. */
typedef struct mag_nersc_info {
    int dims[4];                /* DIMENSION_1..4 */
    int two_row;                /* 1: 4D_SU3_GAUGE, 0: 4D_SU3_GAUGE_3x3 */
    int64_t payload_offset;     /* bytes of the header (the payload follows END_HEADER) */
    uint32_t checksum_header;   /* CHECKSUM (0 if absent) */
    uint32_t checksum;          /* sum modulo 2^32 of the payload's 32-bit words in host byte order */
    uint32_t crc32_header;      /* CRC32HASH (0 if absent) */
    uint32_t crc32;             /* CRC-32 (zlib polynomial) of the host-order payload */
    double plaquette_header;    /* PLAQUETTE (0 if absent) */
    double plaquette;           /* avg_plaquette of the links */
    double link_trace_header;   /* LINK_TRACE (0 if absent) */
    double link_trace;          /* avg_real_trace of the links */
} mag_nersc_info;

/* import_config_nersc (field-matrix.h:594-713) into one chain: reads the
   header (DATATYPE, DIMENSION_1..4, CHECKSUM, PLAQUETTE), checks the lattice
   size, loads the payload, checks the word checksum (the links stay untouched
   on a mismatch), rebuilds the third row of two-row files with reunitarize,
   and checks the plaquette against the header to 1e-4 (the links are loaded
   when this last check fails).  info (may be NULL) receives the header and the
   computed digests.  Errors: MAG_ERR_IO, MAG_ERR_FORMAT, MAG_ERR_CHECKSUM,
   MAG_ERR_PLAQUETTE (the reference asserts instead). */
int mag_gauge_load_nersc(mag_ctx* ctx, int chain, const char* path, mag_nersc_info* info);
/* export_config_nersc (field-matrix.h:452-572) of one chain with Arg_export
   (beta, sequence_num, ensemble_label, field-matrix.h:445-450); two_row =
   doesSkipThird.  CHECKSUM is the word sum of the host-order payload, the value
   import_config_nersc checks; CRC32HASH the CRC-32 of the host-order payload. */
int mag_gauge_save_nersc(mag_ctx* ctx, int chain, const char* path, int two_row, double beta,
                         int sequence_number, const char* ensemble_label, mag_nersc_info* info);
/* header only, no device work (computed fields are 0) */
int mag_nersc_read_header(const char* path, mag_nersc_info* info);

/* --------------------------------------------------- domain decomposition */
/* One lattice split along x3 into nshards slabs of dims[3] / nshards time
   slices (replaces qlat's expanded Geometry and fetch_expanded_chart,
   field-hmc.h:777-781 and :544-558, which run_chmc and
   force_gradient_integrator call before every force; the kinetic, plaquette
   and rectangle sums of get_hamiltonian are added over the slabs as by its
   MPI_Allreduce, field-hmc.h:628, and every slab takes the accept decision
   from the same sums and uniform, as the MPI_Bcast of :823 ensures).  Each
   slab is a context over its time slices plus `halo` slices of each
   neighbour; the halos are refreshed wherever a kernel reads across the
   boundary (the links of each force evaluation, every stout level, the
   double links, each level's Lambda, and the links of the Hamiltonian's
   smearing).  The shards live on the current device and are driven by one
   host thread each.  Requirements: dims[3] % nshards == 0; 2 <= halo <=
   dims[3] / nshards; dims[3] / nshards a multiple of mag (constrained
   segments stay inside one slab); dims[0] dims[1] dims[2] a multiple of 32.
   Results equal the undivided context's up to the order of the global sums
   (MAG_ERR_STATE if the slabs ever disagree on the accept step). */
typedef struct mag_dd mag_dd;
int mag_dd_create(const mag_params* p, int nshards, int halo, mag_dd** out);
int mag_dd_destroy(mag_dd* dd);
/* the lattice's links / momenta in the host layout of mag_gauge_set (every slab
   takes its slices and its halos) and back (every slab gives its own slices) */
int mag_dd_gauge_set(mag_dd* dd, const double* host);
int mag_dd_gauge_get(mag_dd* dd, double* host);
int mag_dd_momentum_set(mag_dd* dd, const double* host);
int mag_dd_momentum_get(mag_dd* dd, double* host);
/* the Philox hot start and uniforms of the undivided lattice (site indices of the whole lattice) */
int mag_dd_hot_start(mag_dd* dd, uint64_t seed);
int mag_dd_uniforms_set(mag_dd* dd, const double* u);
/* get_force (field-hmc.h:339-425) of the whole lattice, halo exchanges included */
int mag_dd_gauge_force(mag_dd* dd, double* host_force);
/* one run_chmc trajectory (field-hmc.h:806-843) of the whole lattice */
int mag_dd_trajectory(mag_dd* dd, int refresh_momenta, mag_traj_result* result);
/* the context of slab `rank` (its time slices are [rank, rank + 1) dims[3] / nshards) */
int mag_dd_shard(mag_dd* dd, int rank, mag_ctx** ctx);

/* One slab per process (or thread), the halos moved by the caller (MPI, NCCL,
   gloo), as qlat's fetch_expanded_chart moves them through MPI.
   mag_shard_create makes the context of slab `rank` (same requirements as
   mag_dd_create); mag_set_halo_fn installs the callback, after which every call
   of the context that reads across the slab boundary or forms the
   Hamiltonian's sums (force, integration, trajectory, Hamiltonian) invokes it,
   every slab in the same order.  Host fields passed to mag_gauge_set and the
   like are the slab's own layout: its dims[3] / nshards + 2 halo time slices,
   lattice time slice rank * dims[3] / nshards - halo first (periodically).
   Trajectories run eagerly (mag_trajectory), not as captured graphs. */
enum { MAG_HALO_EXCHANGE = 0, MAG_HALO_SUM = 1 };
typedef struct mag_halo_op {
    int kind;            /* MAG_HALO_EXCHANGE or MAG_HALO_SUM */
    int rank, nshards;   /* this slab; neighbours are (rank -+ 1) mod nshards */
    /* MAG_HALO_EXCHANGE: a device field of nplanes planes, plane p at base + p * plane_bytes.
       In every plane send the slab_bytes at send_lo to the lower neighbour (it stores them at
       its recv_hi) and those at send_hi to the upper neighbour (its recv_lo); receive the
       lower neighbour's send_hi bytes at recv_lo and the upper neighbour's send_lo bytes at
       recv_hi.  Offsets are bytes within a plane.  The field was produced by work on `stream`
       (a cudaStream_t): order the transfers after it, and make later work on `stream` see the
       received bytes (e.g. NCCL send/recv on `stream`, or synchronise it around host copies). */
    void* base;
    int nplanes;
    size_t plane_bytes, slab_bytes, send_lo, send_hi, recv_lo, recv_hi;
    /* MAG_HALO_SUM: replace sums[0 .. nsums) (host doubles) by their sums over all slabs and,
       when maxval is not NULL, *maxval by its maximum over all slabs */
    double* sums;
    int nsums;
    double* maxval;
    void* stream;
} mag_halo_op;
/* returns 0 on success; any other value makes the calling entry point fail with MAG_ERR_STATE */
typedef int (*mag_halo_fn)(void* user, const mag_halo_op* op);
int mag_shard_create(const mag_params* p, int nshards, int rank, int halo, mag_ctx** out);
int mag_set_halo_fn(mag_ctx* ctx, mag_halo_fn fn, void* user);

/* ---------------------------------------------------- two-level coupling */
/* run_hmc_multi (field-multi.h:758-900): a fine lattice (dims of `fine`, all
   even) and a coarse lattice of half the extent in every direction, coupled
   through the stout-smeared blocked links of the fine field:
     H = K_fine + K_coarse + S_gauge(fine)
         - 1/eta_sqr sum_{coarse x, mu} ReTr(C(x,mu)^dag e^{iQ(2x,mu)} V(2x,mu)),
     V(y,mu) = U(y,mu) U(y+mu,mu) (get_U), Q = -i rho TA(stp V^dag) with stp the
     staple of the 2-link (get_Q, get_staple_rect, field-hmc.h:244-258).
   Forces: get_Fforce (field-multi.h:409-656) and get_Cforce (:659-683); one
   force-gradient trajectory moves both fields (force_gradient_integrator_multi,
   :685-756).  The reference reads rho and eta_sqr from globals that are not in
   its tree; here they are arguments.  Both fields are unconstrained (mag is
   ignored), FP64, no stout levels of the fine action itself.  Fields cross in
   the host layout of mag_gauge_set, fine then coarse. */
typedef struct mag_multi mag_multi;
int mag_multi_create(const mag_params* fine, double rho, double eta_sqr, mag_multi** out);
int mag_multi_destroy(mag_multi* m);
int mag_multi_gauge_set(mag_multi* m, const double* fine, const double* coarse);
int mag_multi_gauge_get(mag_multi* m, double* fine, double* coarse);
int mag_multi_momentum_set(mag_multi* m, const double* fine, const double* coarse);
/* fine force (gauge + coupling) and coarse force of the current fields */
int mag_multi_forces(mag_multi* m, double* fine_force, double* coarse_force);
/* out = {H, kinetic energy of both levels, fine gauge action, coupling energy} */
int mag_multi_hamiltonian(mag_multi* m, double out[4]);
/* one trajectory from the momenta set by mag_multi_momentum_set: Metropolis with
   `uniform` (accepted whatever Delta H while traj_index < n_forced_accept);
   out = {H_old, H_new, Delta H, accept, reunitarisation deviation fine, coarse} */
int mag_multi_trajectory(mag_multi* m, int traj_index, double uniform, double out[6]);

/* ------------------------------------------------------- allocation-free */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc
   (a driver that hands this library memory from a device pool it manages
   itself, or a loop that must not pay for cudaMalloc's implicit device
   synchronisation): the plaquette and rectangle sums of total_plaq /
   total_rectangular (field-matrix.h:299-385), d_sums[0] = sum ReTr plaquette,
   d_sums[1] = sum ReTr rectangle, from links already in device memory in the
   AoS layout double[V][4][3][3][2].  Both pointers are device memory owned by
   the caller; the call only enqueues work on `stream` (a cudaStream_t, NULL =
   default stream) and returns.  It allocates nothing: its block partials live
   in one static device array of MAG_NOALLOC_MAX_SITES / 256 * 2 double-double
   entries (2 MiB), held by every GPU that loads the library until exit, and
   lattices larger than MAG_NOALLOC_MAX_SITES sites are rejected with
   MAG_ERR_ARG.  The first call on a device looks up that array's address
   (again when it is called under another context of that device); make that
   first call before any stream capture.  Calls share the array, so calls that
   overlap on the GPU race with each other.  Like every mag_ctx, it does not
   survive cudaDeviceReset of its device within one process. */
#define MAG_NOALLOC_MAX_SITES (1 << 24)
int mag_action_sums_noalloc(const int dims[4], const double* d_links, double* d_sums, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MAG_C_H */
