"""Error of the mixed-precision path against the plain FP64 path.

    python -m mag_b200.validate --dims 32 32 32 32 --n-stout 3 --steps 16 --therm 6 --samples 4

Both contexts start from the same thermalised FP64 configuration and draw the
same Philox momenta, so every difference below is the precision's:
  * force: |F_mixed - F_fp64| / |F_fp64| (Frobenius over all links) and the
    largest per-link difference relative to the largest force component;
  * Delta H: per trajectory (same U, same P, accept forced by a zero
    uniform), |dH_mixed - dH_fp64|, next to |dH_fp64|;
  * plaquette: after each of those trajectories;
  * reversibility: integrate, flip P, integrate again; max |U_back - U_0| and
    |H_back - H_0| for both precisions (the reunitarisation at the end of each
    integration, field-hmc.h:566, is part of the algorithm and included).
  * with --chain K: K Metropolis trajectories of each precision from the
    thermalised configuration with the same Philox momenta and uniforms: mean
    Delta H, mean exp(-Delta H) (1 at equilibrium), acceptance and plaquette of
    each chain, and how many leading accept decisions the two chains share (while
    they do, their configurations differ only by the precision's rounding).
The FP64 path itself matches the CPU oracle to 1e-11 (force) and 1e-9 (Delta H)
on lattices the oracle can run; this tool extends the comparison to sizes the
oracle cannot.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import mag_b200 as M


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=4, default=[16, 16, 16, 32])
    ap.add_argument("--n-stout", type=int, default=3)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--beta", type=float, default=2.25)
    ap.add_argument("--therm", type=int, default=6, help="forced-accept FP64 trajectories from the hot start")
    ap.add_argument("--samples", type=int, default=4)
    ap.add_argument("--seed", type=int, default=77)
    ap.add_argument("--chain", type=int, default=0,
                    help="also run this many Metropolis trajectories in each precision from the thermalised "
                         "configuration with the same Philox momenta and uniforms, and compare their statistics")
    a = ap.parse_args(argv)
    dims = tuple(a.dims)
    kw = dict(mag=2, action="iwasaki", beta=a.beta, c1=-0.331, rho=0.1, n_stout=a.n_stout, n_steps=a.steps, tau=1.0,
              seed=a.seed)
    out = {"dims": list(dims), "n_stout": a.n_stout, "fg_steps": a.steps, "beta": a.beta}
    with M.Chmc(dims, precision="fp64", n_forced_accept=a.therm, **kw) as c64, \
            M.Chmc(dims, precision="mixed", **kw) as c32:
        c64.hot_start(a.seed)
        if a.therm:
            c64.run_chmc(a.therm)
        U0 = c64.get_gauge()
        c32.set_gauge(U0)
        c64.set_traj_counter(1000)
        c32.set_traj_counter(1000)

        F64, F32 = c64.get_force(), c32.get_force()
        out["force_rel_frobenius"] = float(np.linalg.norm(F32 - F64) / np.linalg.norm(F64))
        out["force_rel_max"] = float(np.abs(F32 - F64).max() / np.abs(F64).max())
        out["force_norm_fp64"] = float(np.linalg.norm(F64))

        rows = []
        for s in range(a.samples):
            r = {}
            for name, c in (("fp64", c64), ("mixed", c32)):
                c.set_gauge(U0)
                c.init_momentum(None, traj=2000 + s)
                c.set_uniforms([0.0])
                (t,) = c.trajectory(refresh_momenta=False)
                r[name] = t
            rows.append({"dH_fp64": r["fp64"]["delta_h"], "dH_mixed": r["mixed"]["delta_h"],
                         "dH_diff": abs(r["mixed"]["delta_h"] - r["fp64"]["delta_h"]),
                         "plaq_fp64": r["fp64"]["avg_plaquette"], "plaq_mixed": r["mixed"]["avg_plaquette"],
                         "plaq_diff": abs(r["mixed"]["avg_plaquette"] - r["fp64"]["avg_plaquette"])})
        out["trajectories"] = rows
        out["dH_diff_max"] = max(x["dH_diff"] for x in rows)
        out["dH_abs_mean_fp64"] = float(np.mean([abs(x["dH_fp64"]) for x in rows]))
        out["plaq_diff_max"] = max(x["plaq_diff"] for x in rows)

        for name, c in (("fp64", c64), ("mixed", c32)):
            c.set_gauge(U0)
            c.init_momentum(None, traj=3000)
            H0, _ = c.get_hamiltonian()
            c.force_gradient_integrator()
            c.init_momentum(-c.get_momentum())
            c.force_gradient_integrator()
            H2, _ = c.get_hamiltonian()
            out[f"reversibility_{name}"] = {"max_dU": float(np.abs(c.get_gauge() - U0).max()),
                                            "abs_dH": abs(H2 - H0)}

        if a.chain:
            seq = {}
            for name, c in (("fp64", c64), ("mixed", c32)):
                c.set_gauge(U0)
                c.set_uniforms(None)
                c.set_traj_counter(5000)
                recs = [r[0] for r in c.run_chmc(a.chain)]
                dh = np.array([r["delta_h"] for r in recs])
                seq[name] = recs
                out[f"chain_{name}"] = {"trajectories": a.chain, "dH_mean": float(dh.mean()),
                                        "dH_abs_mean": float(np.abs(dh).mean()),
                                        "exp_minus_dH_mean": float(np.exp(-dh).mean()),
                                        "acceptance": float(np.mean([r["accept"] for r in recs])),
                                        "plaquette_mean": float(np.mean([r["avg_plaquette"] for r in recs]))}
            same = 0
            for r64, r32 in zip(seq["fp64"], seq["mixed"]):
                if r64["accept"] != r32["accept"]:
                    break
                same += 1
            out["chain_identical_accept_prefix"] = same
            out["chain_dH_diff_max_over_prefix"] = max(
                [abs(r64["delta_h"] - r32["delta_h"]) for r64, r32 in zip(seq["fp64"][:same], seq["mixed"][:same])],
                default=0.0)
            out["chain_plaq_diff_max_over_prefix"] = max(
                [abs(r64["avg_plaquette"] - r32["avg_plaquette"])
                 for r64, r32 in zip(seq["fp64"][:same], seq["mixed"][:same])], default=0.0)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
