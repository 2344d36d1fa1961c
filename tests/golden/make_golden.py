"""Writes the regression fixtures of tests/golden/ from the FP64 oracle.

    python tests/golden/make_golden.py

The reference ships no golden vectors and cannot run here, so these are the
oracle's own outputs on seeded inputs (Philox hot start and momenta), kept so
that a change of the oracle or of the GPU path against them shows up:

* ``hmc_4x4x4x4.npz``: a Haar hot start (seed 3), the Iwasaki force of the thin
  links and through three stout levels (rho = 0.1), the plaquette / rectangle
  sums, and one constrained force-gradient trajectory (8 steps, mag = 2,
  Metropolis) from given momenta and uniform;
* ``unit_2x2x2x4.nersc`` / ``hot_2x2x2x4.nersc``: NERSC files (3x3 and two-row)
  written by the oracle with a fixed ARCHIVE_DATE;
* ``demon_4x4x4x4.npz``: two per-link demon sweeps (E_max = 50, seed 9) of a Haar hot
  start (seed 5): the demon energies after each sweep, the accepted / rejected hit counts,
  the reunitarisation deviations and every 7th site of the swept links.

    python tests/golden/make_golden.py --only demon    # one fixture
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DIMS = (4, 4, 4, 4)
NERSC_DIMS = (2, 2, 2, 4)
ARCHIVE_TIME = 1735689600  # 2025-01-01 00:00:00 UTC


DEMON_SEED, DEMON_SWEEPS, DEMON_EMAX, DEMON_HOT = 9, 2, 50.0, 5


def write_demon() -> None:
    import oracle as O

    U0 = O.gen_hot(DIMS, DEMON_HOT)
    U1, E, acc, rej, dev = O.demon_sweeps(DIMS, U0, seed=DEMON_SEED, n_sweeps=DEMON_SWEEPS, e_max=DEMON_EMAX)
    np.savez_compressed(os.path.join(HERE, "demon_4x4x4x4.npz"), E=E, accepted=acc, rejected=rej, reunit=dev,
                        U_after_every7=U1[::7])


def main(only=None) -> None:
    import oracle as O
    from oracle import nersc as N

    O.build()
    if only == "demon":
        write_demon()
        print("written to", HERE)
        return
    write_demon()
    U = O.gen_hot(DIMS, 3)
    p_thin = O.make_params(DIMS, mag=2, action=1, beta=2.25, n_stout=0, n_steps=8)
    p_st = O.make_params(DIMS, mag=2, action=1, beta=2.25, n_stout=3, rho=0.1, n_steps=8)
    F = O.force(p_thin, U)
    F3 = O.force(p_st, U)
    plaq, rect = O.plaq_rect(DIMS, U)
    P = O.gen_momenta(DIMS, 11, 0)
    u = O.gen_uniform(11, 0)
    U1, rec = O.trajectory(p_thin, 0, U, P, u, [0.0, 0.0])
    np.savez_compressed(
        os.path.join(HERE, "hmc_4x4x4x4.npz"), U=U, F=F, F_stout3=F3, plaq=plaq, rect=rect, P=P, uniform=u,
        U_after=U1, h_old=rec["h_old"], h_new=rec["h_new"], delta_h=rec["delta_h"], accept=rec["accept"],
        avg_plaquette=rec["avg_plaquette"])
    N.export_config(os.path.join(HERE, "unit_2x2x2x4.nersc"), NERSC_DIMS, O.gen_cold(NERSC_DIMS), two_row=False,
                    beta=2.25, seq=1, label="golden", unix_time=ARCHIVE_TIME)
    N.export_config(os.path.join(HERE, "hot_2x2x2x4.nersc"), NERSC_DIMS, O.gen_hot(NERSC_DIMS, 5), two_row=True,
                    beta=2.25, seq=2, label="golden", unix_time=ARCHIVE_TIME)
    print("written to", HERE)


if __name__ == "__main__":
    main(sys.argv[2] if len(sys.argv) > 2 and sys.argv[1] == "--only" else None)
