"""Run force evaluations of one lattice for profiling (e.g. under ncu).

    python -m mag_b200.profile_driver --dims 24 24 24 24 --n-stout 3 --precision fp64 --reps 2

Creates one context, draws a Philox hot start, then times `reps` force
evaluations (plus one warm-up evaluation), optionally `--traj` whole
trajectories, and the named single kernels, and prints the CUDA-event times.  Every launch uses live data, so a profiler that
selects any of them sees a representative kernel.
"""
from __future__ import annotations

import argparse
import json

import mag_b200 as M


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=4, default=[24, 24, 24, 24])
    ap.add_argument("--n-stout", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--action", default="iwasaki", choices=["iwasaki", "wilson"])
    ap.add_argument("--mag", type=int, default=2)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--kernels", nargs="*", default=[])
    ap.add_argument("--no-tune", action="store_true", help="keep the default variants (255-register cap)")
    ap.add_argument("--probe", action="store_true", help="also report the FMA throughput probes")
    ap.add_argument("--demon", type=int, default=0, metavar="SWEEPS",
                    help="also run this many per-link demon sweeps (E_max 50) and report their device time")
    ap.add_argument("--nvtx", action="store_true",
                    help="wrap each --kernels timing loop in an NVTX range time_<kernel> (for ncu --nvtx-include)")
    ap.add_argument("--n-steps", type=int, default=12, help="force-gradient steps per trajectory")
    ap.add_argument("--wilson", type=int, default=0, metavar="RT",
                    help="also time Wilson loops R, T <= RT (inside an NVTX range 'wilson' with --nvtx)")
    ap.add_argument("--ensemble", action="store_true",
                    help="the 96-chain ensemble (48 x 8^4, 32 x 12^4, 16 x 16^4, beta ~ U[2.0, 2.6) from seed 4) "
                         "in place of --dims")
    ap.add_argument("--dd", type=int, default=0, metavar="NSHARDS",
                    help="also time whole trajectories (wall clock, eager) of the lattice split into NSHARDS slabs "
                         "along x3 (halo 2) next to the undivided context's eager trajectories")
    ap.add_argument("--traj", type=int, default=0,
                    help="also run this many trajectories after one warm-up trajectory (inside an NVTX range "
                         "'trajectories' with --nvtx) and report their device time")
    a = ap.parse_args(argv)
    kw = dict(mag=a.mag, action=a.action, n_stout=a.n_stout, rho=0.1, n_steps=a.n_steps, precision=a.precision,
              seed=1)
    if a.ensemble:
        import numpy as np

        rng = np.random.default_rng(4)
        dims = [(8,) * 4] * 48 + [(12,) * 4] * 32 + [(16,) * 4] * 16
        chains = [dict(dims=d, beta=float(b)) for d, b in zip(dims, rng.uniform(2.0, 2.6, len(dims)))]
        ctx = M.Chmc(chains=chains, **kw)
    else:
        ctx = M.Chmc(tuple(a.dims), **kw)
    with ctx as c:
        c.hot_start(1)
        out = {"dims": a.dims, "precision": a.precision, "n_stout": a.n_stout}
        if not a.no_tune:
            out["tuned_min_blocks"] = c.autotune(3)
        out["force_eval_ms"] = c.time_force(a.reps)
        if a.demon:
            res = c.demon_microcanonical(a.demon, 50.0, seed=1)
            out["demon_sweep_ms"] = c.last_measure_ms() / a.demon
            out["demon_accepted"], out["demon_rejected"] = res["accepted"], res["rejected"]
        if a.traj:
            import torch

            c.run_chmc(1)
            torch.cuda.synchronize()
            if a.nvtx:
                torch.cuda.nvtx.range_push("trajectories")
            recs = c.run_chmc(a.traj)
            torch.cuda.synchronize()
            if a.nvtx:
                torch.cuda.nvtx.range_pop()
            out["traj_ms"] = c.last_run_ms() / a.traj
            out["delta_h"] = [r[0]["delta_h"] for r in recs]
        if a.wilson:
            import torch

            c.wilson_loops(a.wilson, a.wilson)
            torch.cuda.synchronize()
            if a.nvtx:
                torch.cuda.nvtx.range_push("wilson")
            ms = []
            for _ in range(a.reps):
                c.wilson_loops(a.wilson, a.wilson)
                ms.append(c.last_measure_ms())
            if a.nvtx:
                torch.cuda.nvtx.range_pop()
            out["wilson_ms"] = sum(ms) / len(ms)
        for k in a.kernels:
            if a.nvtx:
                import torch

                torch.cuda.nvtx.range_push(f"time_{k}")
            out[f"{k}_ms"] = c.time_kernel(k, a.reps)
            if a.nvtx:
                torch.cuda.nvtx.range_pop()
    if a.dd:
        import time

        from mag_b200.dd import DomainChmc

        reps = max(2, a.reps)
        with M.Chmc(tuple(a.dims), **kw) as c:
            c.hot_start(1)
            c.trajectory()
            t0 = time.perf_counter()
            for _ in range(reps):
                c.trajectory()
            t_one = (time.perf_counter() - t0) / reps
        with DomainChmc(tuple(a.dims), a.dd, 2, **kw) as d:
            d.hot_start(1)
            d.trajectory()
            t0 = time.perf_counter()
            for _ in range(reps):
                d.trajectory()
            t_dd = (time.perf_counter() - t0) / reps
        out["dd"] = {"nshards": a.dd, "halo": 2, "undivided_eager_traj_ms": t_one * 1e3,
                     "split_traj_ms": t_dd * 1e3, "ratio": t_dd / t_one}
    if a.probe:
        from mag_b200.field_hmc import probe_fma_peak

        out["fma_tflops"] = {p: probe_fma_peak(p) for p in ("fp64", "fp32", "fp32x2", "fp32x2_selected")}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
