// C++ driver in the style of quench_test/main.C: constrained Iwasaki HMC on a
// hot start through include/mag_field.hpp; prints one JSON line.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "mag_field.hpp"

int main(int argc, char** argv) {
    const int L = argc > 1 ? std::atoi(argv[1]) : 4;
    mag_b200::Arg_chmc arg;
    arg.mag = 2;
    arg.trajectory_length = 4;
    arg.num_trajectory = 3;
    arg.beta = 2.25;
    arg.dt = 1.0 / arg.trajectory_length;
    mag_b200::Options opt;
    opt.n_stout = 1;
    opt.seed = 5;
    try {
        mag_b200::Lattice lat({L, L, L, 2 * L}, arg, opt);
        lat.hot_start(3);
        const double c0 = mag_b200::check_constrained_plaquette(lat);
        std::vector<double> part;
        const double h = mag_b200::get_hamiltonian(lat, part);
        auto res = mag_b200::run_chmc(lat, stderr);
        const double c1 = mag_b200::check_constrained_plaquette(lat);
        // save the configuration and resume from it in a second lattice (quench_test/main.C:92-106)
        double plaq_reload = 0.0;
        if (argc > 2) {
            mag_b200::Arg_export ax;
            ax.beta = arg.beta;
            ax.sequence_num = 3;
            ax.ensemble_label = "cpp_driver";
            mag_b200::export_config_nersc(lat, argv[2], ax, true);
            mag_b200::Lattice lat2({L, L, L, 2 * L}, arg, opt);
            mag_b200::import_config_nersc(lat2, argv[2]);
            plaq_reload = mag_b200::avg_plaquette(lat2);
        }
        // the mass argument m (field-hmc.h:675-693 draws P with width sqrt(m); :427-440 adds F dt m)
        const size_t n = (size_t)lat.volume() * 72;
        std::vector<double> P1(n), P4(n), F(n), Pa(n), Pb(n);
        mag_b200::init_momentum(lat, 7, 1.0);
        mag_b200::check(mag_momentum_get(lat.ctx(), 0, P1.data()), "mag_momentum_get");
        mag_b200::init_momentum(lat, 7, 4.0);
        mag_b200::check(mag_momentum_get(lat.ctx(), 0, P4.data()), "mag_momentum_get");
        int sqrt_m_exact = 1;
        for (size_t i = 0; i < n; i++) sqrt_m_exact &= P4[i] == 2.0 * P1[i];
        mag_b200::get_force(F, lat);
        Pa = P4;
        mag_b200::evolve_momentum(lat, 0.1, 2.5);
        mag_b200::check(mag_momentum_get(lat.ctx(), 0, Pb.data()), "mag_momentum_get");
        double kick_err = 0.0, fmax = 0.0;
        for (size_t i = 0; i < n; i++) {
            kick_err = std::fmax(kick_err, std::fabs(Pb[i] - Pa[i] - 0.25 * F[i]));
            fmax = std::fmax(fmax, std::fabs(F[i]));
        }
        std::printf("{\"h0\": %.17g, \"kin0\": %.17g, \"dh\": [%.17g, %.17g, %.17g], \"plaq\": %.17g, "
                    "\"cplaq_before\": %.17g, \"cplaq_after\": %.17g, \"plaq_reload\": %.17g, "
                    "\"sqrt_m_exact\": %d, \"kick_err\": %.17g, \"fmax\": %.17g}\n",
                    h, part[0], res[0].delta_h, res[1].delta_h, res[2].delta_h, mag_b200::avg_plaquette(lat), c0, c1,
                    plaq_reload, sqrt_m_exact, kick_err, fmax);
    } catch (const mag_b200::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
        return 2;
    }
    return 0;
}
