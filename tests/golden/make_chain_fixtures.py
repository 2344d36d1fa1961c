"""Writes the Markov-chain fixtures of tests/golden/ from the FP64 oracle.

    python tests/golden/make_chain_fixtures.py [--config NAME] [--threads N]

``run_16x16x16x32_3stout.json`` (``--config 16x16x16x32``): the FP64 GPU
configuration at its full size run through the oracle for 20 trajectories:
16^3 x 32, Iwasaki beta = 2.25
(c1 = -0.331), three stout levels rho = 0.1, twelve force-gradient steps of
tau = 1, mag = 2, Metropolis accept, Haar hot start from Philox seed 4,
trajectory t drawing its momenta from ``gen_momenta(dims, 31, t)`` and its
uniform from ``gen_uniform(31, t)`` (the generators the GPU test feeds through
``mag_momentum_set`` / ``mag_uniforms_set``).  Per trajectory it keeps
H_old, H_new, Delta H, the kinetic and action parts, the plaquette and
rectangle sums, the accept bit, the average plaquette and the
reunitarisation deviation; no field is stored (the start and the random
numbers are regenerated from their seeds).

``run_32x32x32x32_3stout.json`` (``--config 32x32x32x32``): the lattice the
mixed-versus-FP64 comparison is stated on, 32^4 with the same action, smearing
and seeds, sixteen force-gradient steps, two trajectories (about 40 minutes
each on 6 threads).

The same run times the oracle's parts (one force evaluation, one link update,
one Hamiltonian) and every whole trajectory on the host's threads, which
checks the trajectory-time extrapolation that the CPU baseline of bench.py
uses (4n force evaluations + 4n + 1 link updates + 2 Hamiltonians).  The run
takes about an hour on 8 threads.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

HOT_SEED, RNG_SEED = 4, 31
PARAMS = dict(mag=2, action=1, beta=2.25, c1=-0.331, rho=0.1, n_stout=3, tau=1.0)
# name: (dims, force-gradient steps, trajectories)
CONFIGS = {"16x16x16x32": ((16, 16, 16, 32), 12, 20), "32x32x32x32": ((32, 32, 32, 32), 16, 2)}
KEYS = ("h_old", "h_new", "delta_h", "kin_old", "kin_new", "pot_old", "pot_new", "plaq_old", "plaq_new",
        "rect_old", "rect_new", "uniform", "reunit_maxdev", "avg_plaquette", "accept")


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="16x16x16x32", choices=sorted(CONFIGS))
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--out", default="")
    a = ap.parse_args()
    import oracle as O

    O.build()
    if a.threads:
        O.set_threads(a.threads)
    DIMS, n_steps, N_TRAJ = CONFIGS[a.config]
    params = dict(PARAMS, n_steps=n_steps)
    out_path = a.out or os.path.join(HERE, f"run_{a.config}_3stout.json")
    po = O.make_params(DIMS, **params)
    U = O.gen_hot(DIMS, HOT_SEED)
    # the parts the CPU baseline extrapolates from, timed on the start configuration
    P = O.gen_momenta(DIMS, RNG_SEED, 0)
    t0 = time.perf_counter()
    O.force(po, U)
    t_force = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.evolve_gauge(po, U, P, 0.01)
    t_evolve = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.hamiltonian(po, U, P)
    t_ham = time.perf_counter() - t0
    n = n_steps
    records, t_traj = [], []
    demon = [0.0, 0.0]
    for t in range(N_TRAJ):
        P = O.gen_momenta(DIMS, RNG_SEED, t)
        u = O.gen_uniform(RNG_SEED, t)
        t0 = time.perf_counter()
        U, r = O.trajectory(po, t, U, P, u, demon)
        t_traj.append(time.perf_counter() - t0)
        demon = r["demon"]
        records.append({k: r[k] for k in KEYS})
        print(f"traj {t}: dH {r['delta_h']:+.6f} accept {r['accept']} plaq {r['avg_plaquette']:.12f} "
              f"({t_traj[-1]:.1f} s)", flush=True)
    out = {
        "dims": list(DIMS), "hot_seed": HOT_SEED, "rng_seed": RNG_SEED, "params": params,
        "accept": "metropolis", "integrator": "force-gradient", "records": records,
        "timing": {"threads": O.lib().mo_get_threads(), "cpu": cpu_model(), "t_force_s": t_force,
                   "t_evolve_s": t_evolve, "t_hamiltonian_s": t_ham,
                   "extrapolated_trajectory_s": 4 * n * t_force + (4 * n + 1) * t_evolve + 2 * t_ham,
                   "measured_trajectory_s": t_traj},
    }
    with open(out_path, "w") as f:
        json.dump(out, f, indent=1)
    print("written", out_path)


if __name__ == "__main__":
    main()
