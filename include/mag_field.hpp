// mag_field.hpp -- C++ drop-in for mag's field-*.h operator names over the C ABI.
//
// A driver written against the reference (quench_test/main.C calling
// run_chmc, field-hmc.h:770) keeps its call structure: the qlat field
// arguments become one mag_b200::Lattice (device-resident links, momenta,
// forces), host configurations cross as AoS double[V][4][3][3][2] buffers.
// Errors throw mag_b200::Error (the reference asserts and aborts).
#ifndef MAG_FIELD_HPP
#define MAG_FIELD_HPP

#include <array>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "mag_c.h"

namespace mag_b200 {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

inline void check(int rc, const char* where) {
    if (rc != MAG_OK) throw Error(rc, std::string(where) + ": " + mag_last_error());
}

// qlat::Gauge (type, c1)
struct Gauge {
    int type = MAG_ACTION_IWASAKI;
    double c1 = -0.331;
};

// Arg_chmc (field-hmc.h:294-307); output directories are the caller's business
struct Arg_chmc {
    int mag = 2;
    int trajectory_length = 12;       // force-gradient steps per trajectory
    int num_trajectory = 20;
    int num_step_between_output = 10;
    int num_forced_accept_step = 0;
    int num_step_before_output = 0;
    double beta = 2.25;
    double dt = 1.0 / 12;             // tau = dt * trajectory_length
    Gauge gauge;
};

// run options that the reference fixes at compile time or leaves undefined
struct Options {
    double rho = 0.1;
    int n_stout = 0;
    int precision = MAG_PREC_FP64;
    int integrator = MAG_INT_FORCE_GRADIENT;
    int accept = MAG_ACCEPT_METROPOLIS;
    double e_max = 100.0;
    uint64_t seed = 1;
};

inline mag_params to_params(const std::array<int, 4>& dims, const Arg_chmc& a, const Options& o) {
    mag_params p{};
    for (int d = 0; d < 4; d++) p.dims[d] = dims[d];
    p.mag = a.mag;
    p.action = a.gauge.type;
    p.beta = a.beta;
    p.c1 = a.gauge.c1;
    p.rho = o.rho;
    p.n_stout = o.n_stout;
    p.tau = a.dt * a.trajectory_length;
    p.n_steps = a.trajectory_length;
    p.precision = o.precision;
    p.integrator = o.integrator;
    p.accept = o.accept;
    p.e_max = o.e_max;
    p.n_forced_accept = a.num_forced_accept_step;
    p.seed = o.seed;
    return p;
}

// The device state of one lattice: gField, mField, fField and the auxiliary
// field of run_chmc (field-hmc.h:777-781) in one object.
class Lattice {
  public:
    Lattice(const std::array<int, 4>& dims, const Arg_chmc& arg, const Options& opt = Options())
        : dims_(dims), arg_(arg) {
        const mag_params p = to_params(dims, arg, opt);
        check(mag_ctx_create(&p, &ctx_), "mag_ctx_create");
    }
    ~Lattice() {
        if (ctx_) mag_ctx_destroy(ctx_);
    }
    Lattice(const Lattice&) = delete;
    Lattice& operator=(const Lattice&) = delete;

    mag_ctx* ctx() const { return ctx_; }
    long volume() const { return (long)dims_[0] * dims_[1] * dims_[2] * dims_[3]; }
    const Arg_chmc& arg() const { return arg_; }

    void set_gauge(const std::vector<double>& aos) { check(mag_gauge_set(ctx_, 0, aos.data()), "mag_gauge_set"); }
    std::vector<double> gauge() const {
        std::vector<double> u((size_t)volume() * 72);
        check(mag_gauge_get(ctx_, 0, u.data()), "mag_gauge_get");
        return u;
    }
    void hot_start(uint64_t seed) { check(mag_gauge_hot_start(ctx_, seed), "mag_gauge_hot_start"); }

  private:
    std::array<int, 4> dims_;
    Arg_chmc arg_;
    mag_ctx* ctx_ = nullptr;
};

// ------------------------------------------------------------ field-hmc.h
// init_momentum (field-hmc.h:675-693): host momenta, or the Philox stream of trajectory `traj`
// with the reference's width sqrt(m) (m = 1 on the HMC path; other m scale on the host)
inline void init_momentum(Lattice& L, const std::vector<double>& P) {
    check(mag_momentum_set(L.ctx(), 0, P.data()), "mag_momentum_set");
}
inline void init_momentum(Lattice& L, uint64_t traj, double m = 1.) {
    check(mag_momentum_refresh(L.ctx(), traj), "mag_momentum_refresh");
    if (m != 1.) {
        std::vector<double> P((size_t)L.volume() * 72);
        check(mag_momentum_get(L.ctx(), 0, P.data()), "mag_momentum_get");
        const double sig = std::sqrt(m);
        for (double& v : P) v *= sig;
        check(mag_momentum_set(L.ctx(), 0, P.data()), "mag_momentum_set");
    }
}

// get_force (field-hmc.h:339-425) into a host AoS buffer
inline void get_force(std::vector<double>& F, Lattice& L) {
    F.resize((size_t)L.volume() * 72);
    check(mag_gauge_force(L.ctx(), 0, F.data()), "mag_gauge_force");
}
// evolve_momentum (field-hmc.h:427-440) with the force of the current links: P += F dt m
inline void evolve_momentum(Lattice& L, double dt, double m = 1.) {
    check(mag_evolve_momentum(L.ctx(), dt * m), "mag_evolve_momentum");
}
// evolve_gauge_field (field-hmc.h:442-482)
inline void evolve_gauge_field(Lattice& L, double dt) { check(mag_evolve_gauge(L.ctx(), dt), "mag_evolve_gauge"); }
// force_gradient_integrator (field-hmc.h:525-567)
inline void force_gradient_integrator(Lattice& L) { check(mag_integrate(L.ctx()), "mag_integrate"); }
// get_hamiltonian (field-hmc.h:589-644): part = {kinetic, potential}
inline double get_hamiltonian(Lattice& L, std::vector<double>& part) {
    double out[3];
    check(mag_hamiltonian(L.ctx(), 0, out), "mag_hamiltonian");
    part.assign({out[1], out[2]});
    return out[0];
}

// ---------------------------------------------------------- field-matrix.h
inline double total_plaq(Lattice& L) {
    double p, r, s;
    check(mag_action(L.ctx(), 0, &p, &r, &s), "mag_action");
    return p;
}
inline double total_rectangular(Lattice& L) {
    double p, r, s;
    check(mag_action(L.ctx(), 0, &p, &r, &s), "mag_action");
    return r;
}
// expiQ (field-hmc.h:82-123) of n Hermitian traceless matrices stored as cps::Matrix
// (18 doubles each, row-major re/im): out[i] = exp(i Q[i])
inline void expiQ(const double* Q, double* out, long n = 1) { check(mag_expiq(Q, n, out), "mag_expiq"); }

// DexpiQ (field-multi.h:90-178) of n pairs (Q, DQ), cps::Matrix layout
inline void DexpiQ(const double* Q, const double* DQ, double* out, long n = 1) {
    check(mag_dexpiq(Q, DQ, n, out), "mag_dexpiq");
}

// compute_Lambda (field-multi.h:180-269) of n triples (Q, Sigma', U), cps::Matrix layout
inline void compute_Lambda(const double* Q, const double* SigmaP, const double* U, double* Lambda, long n = 1) {
    check(mag_compute_lambda(Q, SigmaP, U, n, Lambda), "mag_compute_lambda");
}

inline double avg_plaquette(Lattice& L) {
    double v;
    check(mag_plaquette(L.ctx(), 0, &v), "mag_plaquette");
    return v;
}
inline double reunitarize(Lattice& L) {
    double d;
    check(mag_reunitarize(L.ctx(), &d), "mag_reunitarize");
    return d;
}
inline double check_constrained_plaquette(Lattice& L) {
    double v;
    check(mag_constrained_plaquette(L.ctx(), 0, &v), "mag_constrained_plaquette");
    return v;
}

// ----------------------------------------------------------- field-wloop.h
inline double avg_wilson_loop(Lattice& L, const std::array<int, 3>& r, int T) {
    double v;
    check(mag_wilson_loop(L.ctx(), 0, r.data(), T, &v), "mag_wilson_loop");
    return v;
}

// ------------------------------------------------------------ field-demon.h
// demon_microcanonical (field-demon.h:25-126): arg.num_trajectory sweeps of the
// per-link demons over a copy of the links (the lattice keeps its links).  When
// `summary` is given, the four demon energies of sweep i are appended to it as
// doubles for i >= num_step_before_output and i % num_step_between_output == 0, the
// record the reference writes to demon_equil<info>.dat.  Returns the energies of
// every sweep (4 per sweep).
inline std::vector<double> demon_microcanonical(Lattice& L, double E_max, uint64_t seed = 1,
                                                FILE* summary = nullptr, int64_t* accepted = nullptr,
                                                int64_t* rejected = nullptr) {
    const int n = L.arg().num_trajectory;
    std::vector<double> E((size_t)4 * n);
    std::vector<double> dev((size_t)n);
    check(mag_demon_microcanonical(L.ctx(), 0, n, E_max, seed, 0, E.data(), accepted, rejected, dev.data()),
          "demon_microcanonical");
    if (summary) {
        const int every = L.arg().num_step_between_output > 0 ? L.arg().num_step_between_output : 1;
        for (int i = 0; i < n; i++)
            if (i >= L.arg().num_step_before_output && i % every == 0)
                std::fwrite(E.data() + 4 * i, sizeof(double), 4, summary);
        std::fflush(summary);
    }
    return E;
}

// ---------------------------------------------------- field-matrix.h NERSC I/O
// Arg_export (field-matrix.h:445-450)
struct Arg_export {
    double beta = 0.0;
    int sequence_num = 0;
    std::string ensemble_label;
};
// export_config_nersc (field-matrix.h:452-572); the file is written from the device links
inline mag_nersc_info export_config_nersc(Lattice& L, const std::string& path, const Arg_export& arg,
                                          bool doesSkipThird = false) {
    mag_nersc_info info;
    check(mag_gauge_save_nersc(L.ctx(), 0, path.c_str(), doesSkipThird ? 1 : 0, arg.beta, arg.sequence_num,
                               arg.ensemble_label.c_str(), &info),
          "export_config_nersc");
    return info;
}
// import_config_nersc (field-matrix.h:594-713); throws where the reference asserts
inline mag_nersc_info import_config_nersc(Lattice& L, const std::string& path) {
    mag_nersc_info info;
    check(mag_gauge_load_nersc(L.ctx(), 0, path.c_str(), &info), "import_config_nersc");
    return info;
}

// ------------------------------------------------------------- run_chmc
// run_chmc (field-hmc.h:770-904): arg.num_trajectory trajectories, one summary
// row per trajectory in the reference's format (field-hmc.h:862-864):
// traj, |dH|, exp(-dH), <plaq>, accept, S_gauge.
inline std::vector<mag_traj_result> run_chmc(Lattice& L, FILE* summary = nullptr) {
    const int n = L.arg().num_trajectory;
    std::vector<mag_traj_result> res((size_t)n);
    check(mag_run(L.ctx(), n, res.data()), "mag_run");
    if (summary) {
        int na = 0;
        for (int i = 0; i < n; i++) {
            const mag_traj_result& r = res[i];
            na += r.accept;
            std::fprintf(summary, "%i\t%.6e\t%.6e\t%.12e\t%i\t%.12e\n", r.traj + 1, std::fabs(r.delta_h),
                         std::exp(-r.delta_h), r.avg_plaquette, r.accept, r.accept ? r.action_new : r.action_old);
        }
        std::fprintf(summary, "Accept Rate = %.4f\n", n ? (double)na / n : 0.0);
        std::fflush(summary);
    }
    return res;
}

}  // namespace mag_b200

#endif  // MAG_FIELD_HPP
