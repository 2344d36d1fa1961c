#!/usr/bin/env python
"""Benchmark of the B200 constrained SU(3) HMC path (one JSON line on rank 0).

A step is one HMC trajectory of the workload (momentum refresh, H_old, the
force-gradient molecular dynamics, reunitarisation, H_new, accept/reject),
replayed as one CUDA graph; for the ensemble workload a step advances every
chain by one trajectory and `value` counts chain-trajectories.  The default
workload is the 32^4 lattice, Iwasaki beta = 2.25 (c1 = -0.331), three stout
levels rho = 0.1, sixteen force-gradient steps of tau = 1, constraint
magnification 2, Metropolis accept: `value` is the plain FP64 path and the
same lattice in mixed precision is measured beside it (`mixed`, with its
speed-up over FP64).  On one GPU the default run also measures the 8^4 thin-link
demon configuration, the 16^3 x 32 FP64 configuration (12 FG steps), the 96-chain
ensemble and the 48^3 x 96 mixed configuration with Wilson loops (3 trajectories)
as sub-keys.

  python bench.py [--gpus N --steps K --warmup W] [--workload NAME] [--impl reference]

With --gpus N > 1 (launched by torchrun) every rank advances its own
independent chain(s) on its own GPU: replicas, weak scaling, no collective in
the data path (the only collective is the max over ranks of the timing).

--impl reference times the reference's algorithm on the host cores: the
reference itself cannot be built here (it needs CPS, Qlattice, QMP, MPI), so
this is the FP64 CPU restatement in oracle/ (OpenMP over sites, as the
reference's field-hmc.h:385).  Each of its steps is one full-lattice force
evaluation (the unit a trajectory repeats 4n times); `ms_per_step` is that
timed unit and `value` the trajectory rate extrapolated from it, labelled as
such in `value_basis`.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HMC traj/s & force site-updates/s, mixed vs FP64 GPU at equal ΔH/plaquette"


def ensemble_chains(seed: int = 4):
    """96 independent chains: 48 x 8^4, 32 x 12^4, 16 x 16^4, beta uniform in [2.0, 2.6) from seed."""
    import numpy as np

    rng = np.random.default_rng(seed)
    dims = [(8,) * 4] * 48 + [(12,) * 4] * 32 + [(16,) * 4] * 16
    return [dict(dims=d, beta=float(b)) for d, b in zip(dims, rng.uniform(2.0, 2.6, len(dims)))]


WORKLOADS = {
    # 16^3 x 32, 3 stout levels, 12 FG steps, FP64 (the FP64 GPU path checked against the CPU oracle)
    "16x16x16x32_iwasaki_3stout": dict(dims=(16, 16, 16, 32), beta=2.25, n_stout=3, n_steps=12, precision="fp64"),
    # 32^4, 3 stout levels, 16 FG steps: FP64 with the mixed-precision leg beside it
    "32x32x32x32_iwasaki_3stout": dict(dims=(32, 32, 32, 32), beta=2.25, n_stout=3, n_steps=16, precision="fp64"),
    # 8^4 thin-link Iwasaki, 8 FG steps, demon accept with the demons started at 0 (the CPU-runnable
    # configuration); E_max = 1e5 in units of sum ReTr lets the demons absorb the action change of a hot
    # start (about 7e3 on the first trajectories; with the default 100 every trajectory is rejected)
    "8x8x8x8_iwasaki_thin": dict(dims=(8, 8, 8, 8), beta=2.25, n_stout=0, n_steps=8, precision="fp64",
                                 accept="demon", e_max=1e5),
    # 96 chains in one context, 1 stout level, 8 FG steps, mixed precision
    "ensemble_96chains": dict(chains="ensemble", n_stout=1, n_steps=8, precision="mixed"),
    # 48^3 x 96, beta 2.37, 3 stout levels, 16 FG steps, mixed, Wilson loops R, T <= 8 after each trajectory
    "48x48x48x96_iwasaki_3stout_wloops": dict(dims=(48, 48, 48, 96), beta=2.37, n_stout=3, n_steps=16,
                                             precision="mixed", wilson=8),
    # NERSC configuration load (import_config_nersc) of a 32^4 4D_SU3_GAUGE_3x3 file (604 MB payload);
    # a step is one load from the page cache; the save (export_config_nersc) is timed beside it
    "nersc_io_32x32x32x32": dict(dims=(32, 32, 32, 32), beta=2.25, n_stout=0, n_steps=1, precision="fp64",
                                 kind="nersc"),
    # per-link demon microcanonical sweeps (demon_microcanonical) of an 8^4 hot start, E_max = 50;
    # a step is one sweep over the 16384 links (sequential by definition)
    "demon_8x8x8x8": dict(dims=(8, 8, 8, 8), beta=2.25, n_stout=0, n_steps=1, precision="fp64", kind="demon",
                          e_max=50.0),
    # the same sweeps for 148 independent 8^4 chains at once (mag_demon_microcanonical_all, one CTA per chain,
    # one chain per SM); a step is one sweep of every chain
    "demon_ensemble_148x8x8x8x8": dict(dims=(8, 8, 8, 8), nchains=148, beta=2.25, n_stout=0, n_steps=1,
                                       precision="fp64", kind="demon_ensemble", e_max=50.0),
}
DEFAULT = "32x32x32x32_iwasaki_3stout"
COMMON = dict(mag=2, action="iwasaki", c1=-0.331, rho=0.1, tau=1.0, accept="metropolis", integrator="fg")

# algorithmic flops per site of one launch, reference (gather) formulation:
# 3x3 complex product = 198 flop, matrix add = 18 flop
FLOPS_PER_SITE = {
    # extended staple: 12 plaquette + 72 rectangle path products, 25 adds, per link
    "staple": 4 * (84 * 198 + 25 * 18),
    # thin-link force: staple + U A^dag + traceless anti-Hermitian part
    "force": 4 * (85 * 198 + 25 * 18 + 30),
    # stout level: 12 staple products + Omega + Q^2 + exp combination + exp(iQ) U
    "stout_forward": 4 * (15 * 198 + 6 * 18 + 120),
    # Lambda: U Z, Q^2, Q W, W Q, Z exp(iQ), three traces of products
    "stout_lambda": 4 * (5 * 198 + 3 * 66 + 10 * 18 + 150),
    # chain rule: C recomputed (12 products), C^dag Lambda, 6 insertions x 3 products x 3 directions
    "stout_chain": 4 * (67 * 198 + 24 * 18),
}

# flops per site the kernels execute after reassociation, same conventions
# (complex multiply 6, complex add 2): general product 198, two-row SU(3)
# product 132 + 42 for the reconstructed row = 174, Hermitian x general 162
EXECUTED_FLOPS_PER_SITE = {
    # per link: 2 x 3 x (132 + 174 + 18) + 198 for each of the two shared-factor sums,
    # 3 x 4 x (132 + 174 + 36) for plaquettes and nu-extended rectangles
    "staple": 4 * (2 * (3 * 2 * (132 + 174 + 18) + 198) + 3 * 4 * (132 + 174 + 36) + 18),
    "force": 4 * (2 * (3 * 2 * (132 + 174 + 18) + 198) + 3 * 4 * (132 + 174 + 36) + 18 + 198 + 30),
    # 6 staples (132 + 174 + 18), C U^dag, Q^2, exp combination, exp(iQ) U, coefficients
    "stout_forward": 4 * (6 * (132 + 174 + 18) + 198 + 30 + 162 + 144 + 198 + 120),
    "stout_lambda": 4 * (3 * 198 + 3 * 162 + 2 * 144 + 350),
    # per direction: upper D, E (174 each), three Hermitian products, D x inner (216 with the accumulate);
    # lower G (174), three Hermitian products, one general product, U^dag x inner (216)
    "stout_chain": 4 * (3 * ((2 * 174 + 3 * 162 + 216 + 44) + (174 + 3 * 162 + 198 + 216 + 44)) + 36),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-sub", action="store_true", help="skip the other configurations of the default run")
    return ap.parse_args()


def workload_params(name: str) -> dict:
    p = dict(COMMON)
    p.update(WORKLOADS[name])
    if p.get("chains") == "ensemble":
        p["chains"] = ensemble_chains()
    return p


def site_count(dims) -> int:
    v = 1
    for d in dims:
        v *= d
    return v


def total_sites(params) -> int:
    if "chains" in params:
        return sum(site_count(c["dims"]) for c in params["chains"])
    return site_count(params["dims"])


def max_over_ranks(x: float, dist, device: str) -> float:
    """Max of a per-rank scalar over the process group (identity without one)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(rank: int) -> int:
    return 1000 + 7919 * rank


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: str):
        self.index = index
        self.proc = None
        import tempfile

        fd, self.path = tempfile.mkstemp(prefix="mag_clocks_", suffix=".csv")
        os.close(fd)

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as fh:
            lines = fh.readlines()
        os.remove(self.path)
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), util=float(parts[4]),
                                 hw=parts[6], hwt=parts[7], swt=parts[8], swp=parts[9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r["util"] >= 50] or rows
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                          ("swp", "sw_power_cap")):
            if any(r[key].lower().startswith("active") for r in load):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": reasons, "samples": len(load)}


def gpu_index_for_smi() -> str:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if vis:
        return vis.split(",")[0]
    return "0"


# ---------------------------------------------------------------- CPU legs
def oracle_params(params):
    import oracle as O

    dims = params["dims"] if "dims" in params else params["chains"][-1]["dims"]
    beta = params.get("beta", params["chains"][-1]["beta"] if "chains" in params else 2.25)
    return dims, O.make_params(dims, mag=params["mag"], action=1, beta=beta, c1=params["c1"], rho=params["rho"],
                               n_stout=params["n_stout"], tau=params["tau"], n_steps=params["n_steps"])


def cpu_sample(params: dict) -> dict:
    """Time the oracle (FP64, OpenMP) on one force evaluation, one link update
    and one Hamiltonian evaluation of the full lattice; extrapolate to a
    trajectory: 4n forces + (4n+1) link updates + 2 Hamiltonians."""
    import oracle as O

    dims, po = oracle_params(params)
    U = O.gen_hot(dims, 1)
    P = O.gen_momenta(dims, 1, 0)
    t0 = time.perf_counter()
    O.force(po, U)
    t_force = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.evolve_gauge(po, U, P, 0.01)
    t_evolve = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.hamiltonian(po, U, P)
    t_ham = time.perf_counter() - t0
    n = params["n_steps"]
    traj_s = 4 * n * t_force + (4 * n + 1) * t_evolve + 2 * t_ham
    return {"t_force": t_force, "t_evolve": t_evolve, "t_ham": t_ham, "traj_s": traj_s,
            "cores": O.lib().mo_get_threads()}


def cpu_model() -> str:
    """The host CPU's model name (the CPU baseline runs on it)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def extrapolation_check() -> dict | None:
    """Whole oracle trajectories against the extrapolation from their parts, measured on one host
    when the chain fixtures of tests/golden/ were written (16^3 x 32 with 12 FG steps, 32^4 with 16;
    3 stout levels): the factor that the trajectory rate of the CPU legs rests on.  The 32^4 parts
    were timed while other host jobs ran, so its extrapolation is the more pessimistic one."""
    out = {}
    for lat in ("16x16x16x32", "32x32x32x32"):
        path = os.path.join(ROOT, "tests", "golden", f"run_{lat}_3stout.json")
        if not os.path.exists(path):
            continue
        t = json.load(open(path))["timing"]
        meas = statistics.median(t["measured_trajectory_s"])
        out[lat] = {"threads": t["threads"], "cpu": t["cpu"], "measured_trajectory_s_median": meas,
                    "extrapolated_trajectory_s": t["extrapolated_trajectory_s"],
                    "measured_over_extrapolated": meas / t["extrapolated_trajectory_s"],
                    "trajectories": len(t["measured_trajectory_s"])}
    return out or None


def reference_whole_trajectories(args, params, world, dims, U):
    """Lattices whose whole run fits in two minutes of host time: each step is one whole oracle
    trajectory (momentum draw, H_old, the integrator, reunitarisation, H_new, accept), measured."""
    import oracle as O

    po = O.make_params(dims, mag=params["mag"], action=1, beta=params["beta"], c1=params["c1"], rho=params["rho"],
                       n_stout=params["n_stout"], tau=params["tau"], n_steps=params["n_steps"],
                       accept=1 if params.get("accept") == "demon" else 0, e_max=params.get("e_max", 100.0),
                       n_forced=args.warmup)
    demon = [0.0, 0.0]
    ts = []
    for t in range(args.warmup + args.steps):
        P = O.gen_momenta(dims, 1, t)
        u = O.gen_uniform(1, t)
        t0 = time.perf_counter()
        U, r = O.trajectory(po, t, U, P, u, demon)
        dt = time.perf_counter() - t0
        demon = r["demon"]
        if t >= args.warmup:
            ts.append(dt)
    t_traj = statistics.fmean(ts)
    value = 1.0 / t_traj
    lat = "x".join(map(str, dims))
    cores = O.lib().mo_get_threads()
    line = {
        "metric": METRIC, "value": value, "unit": "traj/s", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_traj * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: Philox Haar hot start",
        "config": config_of(args.workload, params, world),
        "step_definition": f"one whole oracle trajectory of the {lat} lattice (measured, not extrapolated)",
        "value_basis": {"kind": "measured whole trajectories", "t_traj_s_each": ts},
        "cpu_baseline": {"value": value, "unit": "traj/s", "cores": cores, "kind": "port", "cpu": cpu_model(),
                         "sample": f"{args.steps} whole trajectories of the {lat} lattice (FP64 oracle port, "
                                   f"{cores} OpenMP threads), after {args.warmup} untimed ones"},
        "e2e": {"value": value, "unit": "traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_arm(args, params, rank: int, world: int):
    """The oracle (FP64, OpenMP over sites on every host thread) on the workload's lattice.  A step
    is one full-lattice force evaluation, the unit a trajectory repeats 4n times; the link update
    and the Hamiltonian (4n + 1 and 2 per trajectory, about 2% of it) are timed once beforehand.
    `ms_per_step` is the timed unit; `value` is the trajectory rate extrapolated from it."""
    if rank != 0:
        return
    import oracle as O

    dims, po = oracle_params(params)
    U = O.gen_hot(dims, 1)
    P = O.gen_momenta(dims, 1, 0)
    t0 = time.perf_counter()
    O.evolve_gauge(po, U, P, 0.01)
    t_evolve = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.hamiltonian(po, U, P)
    t_ham = time.perf_counter() - t0
    n = params["n_steps"]
    nchain = len(params["chains"]) if "chains" in params else 1
    t0 = time.perf_counter()
    O.force(po, U)
    t_est = 4 * n * (time.perf_counter() - t0) + (4 * n + 1) * t_evolve + 2 * t_ham
    if nchain == 1 and t_est * (args.steps + args.warmup) < 120.0:
        return reference_whole_trajectories(args, params, world, dims, U)
    for _ in range(args.warmup):
        O.force(po, U)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.force(po, U)
        ts.append(time.perf_counter() - t0)
    t_force = statistics.fmean(ts)
    traj_s = 4 * n * t_force + (4 * n + 1) * t_evolve + 2 * t_ham
    # ensemble: every chain's trajectory costs (its volume / the sampled volume) of the sampled one
    traj_s_job = traj_s * total_sites(params) / site_count(dims)
    value = nchain / traj_s_job
    lat = "x".join(map(str, dims))
    cores = O.lib().mo_get_threads()
    sample = (f"each step = one {params['n_stout']}-level stout Iwasaki force evaluation of the {lat} lattice "
              f"(FP64 oracle port, {cores} OpenMP threads); trajectory rate extrapolated from it: {4 * n} force "
              f"evaluations + {4 * n + 1} link updates + 2 Hamiltonians"
              + (", scaled by volume to all chains" if nchain > 1 else ""))
    line = {
        "metric": METRIC, "value": value, "unit": "traj/s", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_force * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: Philox Haar hot start",
        "config": config_of(args.workload, params, world),
        "step_definition": f"one full-lattice force evaluation of the {lat} lattice (the timed unit)",
        "value_basis": {"kind": "extrapolated from the timed force evaluations", "force_evals_per_traj": 4 * n,
                        "link_updates_per_traj": 4 * n + 1, "hamiltonians_per_traj": 2,
                        "t_force_s": t_force, "t_force_s_each": ts, "t_link_update_s": t_evolve,
                        "t_hamiltonian_s": t_ham, "trajectory_s": traj_s_job,
                        "check_whole_trajectories": extrapolation_check()},
        "cpu_baseline": {"value": value, "unit": "traj/s", "cores": cores, "kind": "port", "cpu": cpu_model(),
                         "sample": sample},
        "e2e": {"value": value, "unit": "traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "force_evals_per_s": 1.0 / t_force,
        "site_updates_per_s": site_count(dims) / t_force,
    }
    print(json.dumps(line), flush=True)


def config_of(name, params, world, shard=False):
    c = {"workload": name, "action": "iwasaki", "c1": params["c1"], "stout_levels": params["n_stout"],
         "rho": params["rho"], "fg_steps": params["n_steps"], "tau": params["tau"], "mag": params["mag"],
         "precision": params["precision"], "accept": params.get("accept", "metropolis"),
         "parallelism": f"chains split over {world} GPUs" if shard else f"replicas{world}",
         "l2": "working set > 126 MB L2 (links, momenta, stout levels)"}
    if "chains" in params:
        c["chains"] = "48x8^4 + 32x12^4 + 16x16^4, beta ~ U[2.0, 2.6) per chain"
        c["sites"] = total_sites(params)
    else:
        c["lattice"] = "x".join(str(d) for d in params["dims"])
        c["beta"] = params["beta"]
    if params.get("wilson"):
        c["wilson_loops"] = f"R, T <= {params['wilson']} after each trajectory (FP64)"
    return c


# ---------------------------------------------------------------- GPU arm
def make_ctx(M, params, seed, precision, n_forced):
    kw = {k: v for k, v in params.items() if k not in ("dims", "chains", "wilson")}
    kw["precision"] = precision
    kw["n_forced_accept"] = n_forced  # the reference forces the first accepts (field-hmc.h:826)
    if "chains" in params:
        return M.Chmc(chains=params["chains"], seed=seed, **kw)
    return M.Chmc(params["dims"], seed=seed, **kw)


def measured_hbm_gbs() -> float:
    """MEASURED_PEAKS.json's copy bandwidth of this pool's B200s, else the earlier measurement 6.65 TB/s."""
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        return float(json.load(open(pp)).get("hbm_gbs", 6650.0))
    return 6650.0


def wilson_bytes(wl: int, V: int) -> int:
    """Algorithmic HBM bytes of one Wilson-loop measurement (R, T <= wl, three spatial directions) of V
    sites: per direction the R-line planes (first: read U, write the line; then read U and the previous
    line, write), per T the temporal line (the same) and the accumulation pass (reads the wl S-line
    planes and the temporal line once per site; the shifted reads come from L2)."""
    per_dir = (288 + (wl - 1) * 432) + (288 + (wl - 1) * 432) + wl * (wl + 1) * 144
    return 3 * per_dir * V


def sub_run(M, workload: str, precisions, args, steps: int | None = None, warmup: int | None = None) -> dict:
    """One GPU, no collective: W forced-accept trajectories, then K timed ones (CUDA events around
    the graph launches) per precision; chain-trajectories/s for an ensemble.  A workload with Wilson
    loops measures them after every timed trajectory, inside the timed total."""
    import torch

    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    params = workload_params(workload)
    wl = params.get("wilson", 0)
    nchain = len(params["chains"]) if "chains" in params else 1
    out = {"workload": workload, "fg_steps": params["n_steps"], "stout_levels": params["n_stout"]}
    if "chains" in params:
        out["chains"] = nchain
        out["sites"] = total_sites(params)
    else:
        out["lattice"] = "x".join(map(str, params["dims"]))
    for prec in precisions:
        c = make_ctx(M, params, rank_seed(0), prec, warmup)
        dev = c.device_bytes()  # the context's fields, touched by every trajectory
        out["l2"] = (f"working set {dev / 1e9:.2f} GB > 126 MB L2" if dev > 126e6
                     else f"working set {dev / 1e6:.0f} MB inside the 126 MB L2 (no flush between trajectories)")
        c.hot_start(rank_seed(0))
        if warmup:
            c.run_chmc(warmup)
        torch.cuda.synchronize()
        wl_ms = 0.0
        if wl:
            recs, ms = [], 0.0
            for _ in range(steps):
                recs += c.run_chmc(1)
                ms += c.last_run_ms()
                c.wilson_loops(wl, wl)
                wl_ms += c.last_measure_ms()
        else:
            recs = c.run_chmc(steps)
            ms = c.last_run_ms()
        out[prec] = {"value": nchain * steps / ((ms + wl_ms) / 1e3),
                     "unit": "chain-traj/s" if nchain > 1 else "traj/s", "ms_per_step": (ms + wl_ms) / steps,
                     "steps": steps, "warmup": warmup,
                     "acceptance": statistics.fmean(r[k]["accept"] for r in recs for k in range(nchain)),
                     "delta_h_mean": statistics.fmean(r[k]["delta_h"] for r in recs for k in range(nchain)),
                     "plaquette": recs[-1][0]["avg_plaquette"],
                     "graph_kernels_per_step": c.graph_kernel_count()}
        if wl:
            out[prec]["wilson_loops_ms_per_step"] = wl_ms / steps
            out[prec]["wilson_share_of_step"] = wl_ms / (ms + wl_ms)
            hbm = measured_hbm_gbs()
            wach = wilson_bytes(wl, total_sites(params)) / (wl_ms / steps * 1e-3) / 1e9
            out[prec]["wilson_hbm"] = {"achieved": wach, "peak": hbm, "unit": "GB/s", "frac": wach / hbm,
                                       "bytes_per_measurement": wilson_bytes(wl, total_sites(params))}
        c.close()
    if "fp64" in out and "mixed" in out:
        out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def run_gpu(args, params, rank, world, dist):
    import numpy as np
    import torch

    import mag_b200 as M
    from mag_b200.field_hmc import probe_fma_peak

    n = params["n_steps"]
    full_params = params
    # an ensemble on N > 1 GPUs is split over the ranks (balanced by V x steps), each chain
    # keeping its Philox stream; a single lattice runs as N independent replicas
    shard = "chains" in params and world > 1
    parts = None
    if shard:
        from mag_b200.ensemble import chain_cost, partition

        parts = partition([chain_cost(ch["dims"], n) for ch in params["chains"]], world)
        params = dict(params)
        params["chains"] = [full_params["chains"][i] for i in parts[rank]]
    V = total_sites(params)
    nchain = len(params["chains"]) if "chains" in params else 1
    job_chains = len(full_params["chains"]) if shard else world * nchain  # chains advanced per step, all ranks
    job_sites = total_sites(full_params) if shard else world * V
    seed = rank_seed(0) if shard else rank_seed(rank)
    wl = params.get("wilson", 0)

    def timed_run(prec: str):
        c = make_ctx(M, params, seed, prec, args.warmup)
        if shard:
            c.set_stream_index(parts[rank])
        c.hot_start(seed)
        if args.warmup:
            c.run_chmc(args.warmup)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(gpu_index_for_smi()) if rank == 0 else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        recs, ms, wl_ms = [], 0.0, 0.0
        if wl:
            for _ in range(args.steps):
                recs += c.run_chmc(1)
                ms += c.last_run_ms()
                c.wilson_loops(wl, wl)
                wl_ms += c.last_measure_ms()
        else:
            recs = c.run_chmc(args.steps)
            ms = c.last_run_ms()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        total = max_over_ranks(ms + wl_ms, dist, "cuda")
        return c, recs, total, wl_ms, clocks

    head_prec = params["precision"]
    c64, rec64, ms64, wl_ms, clocks = timed_run(head_prec)
    value = job_chains * args.steps / (ms64 / 1e3)
    ms_per_step = ms64 / args.steps
    if shard:
        from mag_b200.ensemble import gather_records

        rec64 = gather_records(rec64, parts, rank, dist, "cuda")  # every rank, same shapes
    nrec = len(rec64[0])
    dh = [r[k]["delta_h"] for r in rec64 for k in range(nrec)]
    acc = [r[k]["accept"] for r in rec64 for k in range(nrec)]
    plaq = rec64[-1][0]["avg_plaquette"]
    kernels_per_traj = c64.graph_kernel_count()

    # dominant kernel and its roofline (device-timed on the launching stream)
    names = ["staple", "stout_forward", "stout_lambda", "stout_chain"] if params["n_stout"] else ["force"]
    per_eval = {"staple": 1, "force": 1, "stout_forward": params["n_stout"], "stout_lambda": params["n_stout"],
                "stout_chain": params["n_stout"]}
    kt = {k: c64.time_kernel(k, 5) for k in names}
    share = {k: kt[k] * per_eval[k] for k in names}
    dom = max(share, key=share.get)
    t_force_eval = c64.time_force(3)
    prec_key = "fp64" if head_prec == "fp64" else "fp32"
    peak = probe_fma_peak(prec_key)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(f"{args.workload}:{head_prec}:{dom}")
    # achieved = flops the kernel executes per launch (two-row SU(3) and Hermitian products, confirmed
    # by ncu's FMA/ADD/MUL instruction counts) / its CUDA-event launch time
    executed = EXECUTED_FLOPS_PER_SITE[dom] * V / (kt[dom] * 1e-3) / 1e12
    gather = FLOPS_PER_SITE[dom] * V / (kt[dom] * 1e-3) / 1e12
    roofline = {"bound": prec_key, "kernel": dom, "achieved": executed, "peak": peak, "unit": "TFLOP/s",
                "frac": executed / peak, "traffic": traffic, "flops_per_site": EXECUTED_FLOPS_PER_SITE[dom],
                "algorithmic_equiv": {"achieved": gather, "frac": gather / peak, "flops_per_site": FLOPS_PER_SITE[dom],
                                      "note": "the reference's gather formulation (85 / 67 products per link); "
                                              "the kernels execute fewer flops, so this can exceed 1"},
                "peak_source": f"measured CUDA-core {prec_key.upper()} FMA throughput (mag_probe_fma_peak)",
                "launch_ms": kt[dom], "kernel_ms": kt,
                "executed_frac": {k: EXECUTED_FLOPS_PER_SITE[k] * V / (kt[k] * 1e-3) / 1e12 / peak for k in names},
                "force_eval_ms": t_force_eval, "tuned": c64.autotune(3)}
    ev_ms = c64.time_kernel("evolve", 5)
    bytes_evolve = V * 4 * (144 + 144 + 64) + (V * 4 * 72 if head_prec == "mixed" else 0)
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    hbm_peak = measured_hbm_gbs()
    roofline["evolve_hbm"] = {"achieved": bytes_evolve / (ev_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                              "frac": bytes_evolve / (ev_ms * 1e-3) / 1e9 / hbm_peak,
                              "peak_source": ("MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks
                                              else "fallback 6.65 TB/s")}

    # end to end through the public API with pinned host buffers (every chain of this rank's context)
    e2e = None
    if args.e2e_steps > 0:
        nloc = c64.n_chains

        def pinned_field(V):
            return torch.empty(V * 72, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(
                V, 4, 3, 3)

        Uh = [pinned_field(c64.volume(k)) for k in range(nloc)]
        for k in range(nloc):
            c64.get_gauge(k, out=Uh[k])
        rng = np.random.default_rng(seed)
        s2, s6 = 1 / np.sqrt(2), 1 / np.sqrt(6)
        Ps = []  # pinned momentum fields (two sets, used in turn), filled before the timed region
        for _ in range(min(args.e2e_steps, 2)):
            Pset = []
            for k in range(nloc):
                V = c64.volume(k)
                xi = rng.standard_normal((V, 4, 8))
                P = pinned_field(V)
                P[..., 0, 1] = (xi[..., 0] - 1j * xi[..., 1]) * s2
                P[..., 0, 2] = (xi[..., 3] - 1j * xi[..., 4]) * s2
                P[..., 1, 2] = (xi[..., 5] - 1j * xi[..., 6]) * s2
                P[..., 1, 0] = P[..., 0, 1].conj()
                P[..., 2, 0] = P[..., 0, 2].conj()
                P[..., 2, 1] = P[..., 1, 2].conj()
                P[..., 0, 0] = xi[..., 2] * s2 + xi[..., 7] * s6
                P[..., 1, 1] = -xi[..., 2] * s2 + xi[..., 7] * s6
                P[..., 2, 2] = -2 * xi[..., 7] * s6
                Pset.append(P)
            Ps.append(Pset)
        field_bytes = sum(c64.volume(k) for k in range(nloc)) * 4 * 9 * 16
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for j in range(args.e2e_steps):
            for k in range(nloc):
                c64.set_gauge(Uh[k], chain=k)
                c64.init_momentum(Ps[j % len(Ps)][k], chain=k)
            c64.set_uniforms([0.5] * nloc)
            c64.trajectory(refresh_momenta=False)
            if wl:
                c64.wilson_loops(wl, wl)
            for k in range(nloc):
                c64.get_gauge(k, out=Uh[k])
        torch.cuda.synchronize()
        el = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        e2e = {"value": job_chains * args.e2e_steps / el, "unit": "traj/s",
               "h2d_bytes_per_step": 2 * field_bytes + 8 * nloc, "d2h_bytes_per_step": field_bytes + 152 * nloc,
               "steps": args.e2e_steps,
               "path": "mag_gauge_set + mag_momentum_set per chain, mag_uniforms_set, mag_trajectory, "
                       "mag_gauge_get per chain"}
    c64.close()

    mixed = None
    if not args.no_mixed and head_prec == "fp64":
        cm, recm, msm, _, _ = timed_run("mixed")
        vm = job_chains * args.steps / (msm / 1e3)
        mixed = {"value": vm, "unit": "traj/s", "ms_per_step": msm / args.steps, "speedup_vs_fp64": vm / value,
                 "delta_h_mean": statistics.fmean(r[0]["delta_h"] for r in recm),
                 "exp_minus_delta_h_mean": statistics.fmean(math.exp(-r[0]["delta_h"]) for r in recm),
                 "acceptance": statistics.fmean(r[0]["accept"] for r in recm),
                 "plaquette": recm[-1][0]["avg_plaquette"],
                 "force_eval_ms": cm.time_force(3)}
        cm.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        s = cpu_sample(params)
        vol_ratio = V / site_count(oracle_params(params)[0])
        cpu = {"value": nchain / (s["traj_s"] * vol_ratio), "unit": "traj/s", "cores": s["cores"], "kind": "port",
               "cpu": cpu_model(), "extrapolation_check": extrapolation_check(),
               "sample": (f"oracle FP64 port, OpenMP: one force evaluation ({s['t_force']:.2f} s), one link update "
                          f"({s['t_evolve']:.2f} s) and one Hamiltonian ({s['t_ham']:.2f} s) of the "
                          f"{'x'.join(map(str, oracle_params(params)[0]))} lattice, extrapolated to {4 * n} force "
                          f"evals + {4 * n + 1} updates + 2 Hamiltonians per trajectory"
                          + (" and by volume to all chains" if nchain > 1 else "")),
               "force_evals_per_s": 1.0 / s["t_force"]}

    # the other HMC configurations, measured beside the headline on one GPU
    sub = {}
    if world == 1 and args.workload == DEFAULT and not args.no_sub:
        sub["config1_8x8x8x8_thin_demon"] = sub_run(M, "8x8x8x8_iwasaki_thin", ("fp64",), args)
        sub["config2_16x16x16x32"] = sub_run(M, "16x16x16x32_iwasaki_3stout", ("fp64", "mixed"), args)
        sub["ensemble_96chains"] = sub_run(M, "ensemble_96chains", ("mixed",), args)
        # 48^3 x 96 (10.6M sites, 72 GB in mixed precision): 4.4 s per trajectory, so 3 warm-up and 3
        # timed trajectories, each followed by the Wilson loops R, T <= 8
        sub["config5_48x48x48x96_wloops"] = sub_run(M, "48x48x48x96_iwasaki_3stout_wloops", ("mixed",), args,
                                                    steps=min(args.steps, 3), warmup=min(args.warmup, 3))

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "traj/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if shard else "weak",
        "vs_baseline": None, "dtype": "f64" if head_prec == "fp64" else "f32+f64",
        "data": "synthetic: Philox Haar-random hot start, Gaussian momenta, Philox Metropolis uniforms",
        "config": config_of(args.workload, full_params, world, shard),
        "force_evals_per_s": job_chains * 4 * n * args.steps / (ms64 / 1e3),
        "site_updates_per_s": job_sites * 4 * n * args.steps / (ms64 / 1e3),
        "delta_h_mean": statistics.fmean(dh), "delta_h_abs_mean": statistics.fmean(abs(x) for x in dh),
        "exp_minus_delta_h_mean": statistics.fmean(math.exp(-x) for x in dh),
        "acceptance": statistics.fmean(acc), "plaquette": plaq,
        "mixed": mixed, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": kernels_per_traj * args.steps,
    }
    if sub:
        line["other_configs"] = sub
    if wl:
        line["wilson_loops_ms_per_step"] = wl_ms / args.steps
        # HBM roofline of one Wilson-loop measurement (bytes as wilson_bytes counts them)
        wbytes = wilson_bytes(wl, V)
        wach = wbytes / (wl_ms / args.steps * 1e-3) / 1e9
        line["wilson_hbm"] = {"achieved": wach, "peak": hbm_peak, "unit": "GB/s", "frac": wach / hbm_peak,
                              "bytes_per_measurement": wbytes,
                              "share_of_step": wl_ms / (ms64 if ms64 else 1.0)}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- NERSC I/O workload
NERSC_METRIC = "NERSC configuration load throughput (payload GB/s, import_config_nersc)"


def nersc_dir(need_bytes: int) -> str:
    """A scratch directory for the configuration files: /dev/shm when it has room, else the temp dir."""
    import shutil
    import tempfile

    for base in ("/dev/shm", None):
        try:
            d = tempfile.mkdtemp(prefix="mag_nersc_", dir=base)
        except OSError:
            continue
        if shutil.disk_usage(d).free > need_bytes + (1 << 30):
            return d
        shutil.rmtree(d, ignore_errors=True)
    return tempfile.mkdtemp(prefix="mag_nersc_")


def nersc_config(args, params, world):
    return {"workload": args.workload, "lattice": "x".join(str(d) for d in params["dims"]),
            "datatype": "4D_SU3_GAUGE_3x3", "file": "page cache (written just before the timed loads)",
            "parallelism": f"replicas{world}", "l2": "payload 604 MB > 126 MB L2"}


def nersc_reference_arm(args, params, rank: int, world: int):
    """import_config_nersc restated on the host (numpy byte order and digests, the oracle's OpenMP
    plaquette), on the same file; each step is one full load."""
    if rank != 0:
        return
    import shutil

    import oracle as O
    from oracle import nersc as N

    dims = params["dims"]
    B = site_count(dims) * 4 * 9 * 16
    d = nersc_dir(B)
    try:
        path = os.path.join(d, "cfg.nersc")
        N.export_config(path, dims, O.gen_hot(dims, 1), two_row=False, beta=params["beta"])
        for _ in range(args.warmup):
            N.import_config(path, dims)
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            N.import_config(path, dims)
            ts.append(time.perf_counter() - t0)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    t = statistics.median(ts)
    value = B / t / 1e9
    line = {"metric": NERSC_METRIC, "value": value, "unit": "GB/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: Philox Haar hot start",
            "config": nersc_config(args, params, world),
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": O.lib().mo_get_threads(), "kind": "port",
                             "sample": "one import of the 604 MB file per step (numpy byte order, checksum, "
                                       "zlib CRC, OpenMP plaquette)"},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_nersc(args, params, rank, world, dist):
    import shutil

    import torch

    import mag_b200 as M

    dims = params["dims"]
    V = site_count(dims)
    B = V * 4 * 9 * 16
    seed = rank_seed(rank)
    d = nersc_dir(2 * B)
    path = os.path.join(d, "cfg.nersc")
    try:
        with M.Chmc(dims, mag=params["mag"], beta=params["beta"], n_stout=0, seed=seed) as c:
            c.hot_start(seed)
            c.export_config_nersc(path, skip_third=False)
            for _ in range(args.warmup):
                c.import_config_nersc(path)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            sampler = ClockSampler(gpu_index_for_smi()) if rank == 0 else None
            if sampler:
                sampler.start()
                time.sleep(0.3)
            t_load = []
            for _ in range(args.steps):
                t0 = time.perf_counter()
                c.import_config_nersc(path)
                t_load.append(time.perf_counter() - t0)
            t_save = []
            for _ in range(max(1, args.steps // 2)):
                t0 = time.perf_counter()
                c.export_config_nersc(path + ".out", skip_third=False)
                t_save.append(time.perf_counter() - t0)
            kt = {k: c.time_kernel(k, 5) for k in ("nersc_swap", "nersc_crc", "nersc_to_links", "nersc_from_links",
                                                   "nersc_plaq")}
            torch.cuda.synchronize()
            clocks = sampler.stop() if sampler else None
        tl = max_over_ranks(statistics.median(t_load), dist, "cuda")
        ts = max_over_ranks(statistics.median(t_save), dist, "cuda")
        dev_ms = kt["nersc_swap"] + kt["nersc_crc"] + kt["nersc_to_links"] + kt["nersc_plaq"]
        dev_ms = max_over_ranks(dev_ms, dist, "cuda")
    finally:
        shutil.rmtree(d, ignore_errors=True)
    if rank != 0:
        return
    # algorithmic HBM bytes per launch: swap reads + writes the payload, CRC reads it, the
    # conversion reads it and writes the same bytes of link tiles
    abytes = {"nersc_swap": 2 * B, "nersc_crc": B, "nersc_to_links": 2 * B, "nersc_from_links": 2 * B}
    dom = max(("nersc_swap", "nersc_crc", "nersc_to_links"), key=lambda k: kt[k])
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    hbm = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(f"{args.workload}:fp64:{dom}")
    achieved = abytes[dom] / (kt[dom] * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu:
        import oracle as O
        from oracle import nersc as N

        d2 = nersc_dir(B)
        try:
            p2 = os.path.join(d2, "cfg.nersc")
            N.export_config(p2, dims, O.gen_hot(dims, 1), two_row=False, beta=params["beta"])
            t0 = time.perf_counter()
            N.import_config(p2, dims)
            tc = time.perf_counter() - t0
        finally:
            shutil.rmtree(d2, ignore_errors=True)
        cpu = {"value": B / tc / 1e9, "unit": "GB/s", "cores": O.lib().mo_get_threads(), "kind": "port",
               "sample": "one import of the same-size 3x3 file (numpy byte order, checksum, zlib CRC, OpenMP "
                         "plaquette)"}
    line = {
        "metric": NERSC_METRIC, "value": world * B / (dev_ms * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8/f64", "data": "synthetic: Philox Haar hot start",
        "config": nersc_config(args, params, world),
        "value_definition": "payload bytes / device time of the load kernels (byte order + checksum, CRC-32, "
                            "conversion to link tiles, plaquette and link-trace sums), payload already in HBM",
        "kernel_ms": kt,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "algorithmic_bytes": abytes[dom],
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6.65 TB/s"},
        "cpu_baseline": cpu,
        "e2e": {"value": world * B / tl / 1e9, "unit": "GB/s", "h2d_bytes_per_step": B, "d2h_bytes_per_step": 0,
                "path": "mag_gauge_load_nersc from a file in the page cache (read, copy, digests, conversion, "
                        "plaquette check)", "ms_per_step": tl * 1e3},
        "save_e2e": {"value": world * B / ts / 1e9, "unit": "GB/s", "d2h_bytes_per_step": B,
                     "path": "mag_gauge_save_nersc to the page cache", "ms_per_step": ts * 1e3},
        "clocks": clocks,
        "gpu_launches": 8 * args.steps,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- demon sweep workload
DEMON_METRIC = "per-link demon sweeps/s (demon_microcanonical, link updates/s = 4 V sweeps/s)"
# flops of one link: 6 plaquette paths (2 products), 162 five-link paths (4 products), 198 per
# product, and two hits of 3 products on each of 4 demons
DEMON_FLOPS_PER_LINK = (6 * 2 + 162 * 4) * 198 + 2 * 4 * 3 * 198


def demon_config(args, params, world):
    return {"workload": args.workload, "lattice": "x".join(str(d) for d in params["dims"]),
            "e_max": params["e_max"], "hits_per_link": 2, "demons": "plaquette, rectangle, chair, twist",
            "parallelism": f"replicas{world}", "l2": "8^4 links (4.7 MB) stay in L2: one sweep is latency-bound"}


def demon_reference_arm(args, params, rank: int, world: int):
    """The oracle's sequential restatement (one host thread: the sweep is sequential)."""
    if rank != 0:
        return
    import oracle as O

    dims = params["dims"]
    U = O.gen_hot(dims, 1)
    for _ in range(args.warmup):
        O.demon_sweeps(dims, U, 1, 1, params["e_max"])
    ts = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        O.demon_sweeps(dims, U, 1 + i, 1, params["e_max"])
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    line = {"metric": DEMON_METRIC, "value": 1.0 / t, "unit": "sweeps/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: Philox Haar hot start",
            "config": demon_config(args, params, world),
            "cpu_baseline": {"value": 1.0 / t, "unit": "sweeps/s", "cores": 1, "kind": "port",
                             "sample": f"one sweep over the {4 * site_count(dims)} links per step"},
            "e2e": {"value": 1.0 / t, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


DEMON_ENS_METRIC = "per-link demon link updates/s over an ensemble of chains (one CTA per chain)"


def demon_ensemble_config(args, params, world):
    return {"workload": args.workload, "lattice": "x".join(str(d) for d in params["dims"]),
            "chains": params["nchains"], "e_max": params["e_max"], "hits_per_link": 2,
            "demons": "plaquette, rectangle, chair, twist", "parallelism": f"chains x replicas{world}",
            "l2": "148 x 8^4 links (0.7 GB) exceed the 126 MB L2"}


def oracle_ensemble_rate(params, n_chains: int, seed: int):
    """Link updates/s of the oracle sweeping n_chains chains on all host threads, one chain per
    thread (the oracle's sweep releases the interpreter lock)."""
    import concurrent.futures as cf

    import oracle as O

    dims = params["dims"]
    threads = os.cpu_count() or 1
    fields = [O.gen_hot(dims, seed + k) for k in range(n_chains)]
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda k: O.demon_sweeps(dims, fields[k], seed + k, 1, params["e_max"]), range(n_chains)))
    t = time.perf_counter() - t0
    return n_chains * 4 * site_count(dims) / t, threads, t


def demon_ensemble_reference_arm(args, params, rank: int, world: int):
    """The oracle's sweeps of independent chains on all host threads; a step sweeps one chain per thread."""
    if rank != 0:
        return
    n = os.cpu_count() or 1
    for i in range(args.warmup):
        oracle_ensemble_rate(params, 1, 100 + i)
    rates = [oracle_ensemble_rate(params, n, 1 + n * i)[0] for i in range(args.steps)]
    rate = statistics.median(rates)
    step_s = n * 4 * site_count(params["dims"]) / rate
    line = {"metric": DEMON_ENS_METRIC, "value": rate, "unit": "link updates/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: Philox Haar hot starts", "config": demon_ensemble_config(args, params, world),
            "cpu_baseline": {"value": rate, "unit": "link updates/s", "cores": n, "kind": "port",
                             "sample": f"{n} chains swept once per step, one host thread each"},
            "e2e": {"value": rate, "unit": "link updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_demon_ensemble(args, params, rank, world, dist):
    import torch
    import numpy as np

    import mag_b200 as M
    from mag_b200.field_hmc import probe_fma_peak

    dims, n = params["dims"], params["nchains"]
    V = site_count(dims)
    seed = rank_seed(rank)
    with M.Chmc(chains=[dict(dims=dims, beta=params["beta"], mag=0) for _ in range(n)], n_stout=0, seed=seed) as c:
        c.hot_start(seed)
        c.demon_microcanonical_all(args.warmup, params["e_max"], seed=seed)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        sampler = ClockSampler(gpu_index_for_smi()) if rank == 0 else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        torch.cuda.synchronize()
        res = c.demon_microcanonical_all(args.steps, params["e_max"], seed=seed + 1)
        torch.cuda.synchronize()
        dev_s = c.last_measure_ms() / 1e3  # CUDA events on the library's stream around the sweeps
        clocks = sampler.stop() if sampler else None
        # end to end: every chain's links in from pinned host memory, one sweep keeping them, links out
        Uh = [torch.empty(V * 72, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(
            V, 4, 3, 3) for _ in range(n)]
        for k in range(n):
            c.get_gauge(k, out=Uh[k])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for j in range(args.steps):
            for k in range(n):
                c.set_gauge(Uh[k], chain=k)
            c.demon_microcanonical_all(1, params["e_max"], seed=seed + 2 + j, update_links=True)
            for k in range(n):
                c.get_gauge(k, out=Uh[k])
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    el = max_over_ranks(dev_s, dist, "cuda")
    wall = max_over_ranks(wall, dist, "cuda")
    if rank != 0:
        return
    sweep_s = el / args.steps
    links = world * n * 4 * V
    flops = DEMON_FLOPS_PER_LINK * links / world / sweep_s / 1e12
    peak = probe_fma_peak("fp64")
    cpu = None
    if not args.no_cpu:
        rate, threads, tc = oracle_ensemble_rate(params, 2 * (os.cpu_count() or 1), 1)
        cpu = {"value": rate, "unit": "link updates/s", "cores": threads, "kind": "port",
               "sample": f"{2 * threads} chains of {'x'.join(map(str, dims))} swept once, one host thread each "
                         f"({tc:.1f} s)"}
    line = {
        "metric": DEMON_ENS_METRIC, "value": links / sweep_s, "unit": "link updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sweep_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: Philox Haar hot starts",
        "config": demon_ensemble_config(args, params, world),
        "chain_sweeps_per_s": world * n / sweep_s,
        "accepted": int(sum(r["accepted"] for r in res)), "rejected": int(sum(r["rejected"] for r in res)),
        "roofline": {"bound": "fp64 (one CTA per chain, sequential inside a chain)", "achieved": flops,
                     "peak": peak, "unit": "TFLOP/s", "frac": flops / peak, "traffic": None,
                     "flops_per_link": DEMON_FLOPS_PER_LINK,
                     "peak_source": "measured CUDA-core FP64 FMA throughput of the device"},
        "cpu_baseline": cpu,
        "e2e": {"value": world * n * 4 * V * args.steps / wall, "unit": "link updates/s",
                "h2d_bytes_per_step": n * 576 * V, "d2h_bytes_per_step": n * (576 * V + 48 + 8),
                "path": "mag_gauge_set per chain + mag_demon_microcanonical_all (one sweep, links kept) + "
                        "mag_gauge_get per chain, from / to pinned host buffers"},
        "clocks": clocks,
        "gpu_launches": (2 * n + 2) * args.steps,
    }
    print(json.dumps(line), flush=True)


def run_demon(args, params, rank, world, dist):
    import torch
    import numpy as np

    import mag_b200 as M
    from mag_b200.field_hmc import probe_fma_peak

    dims = params["dims"]
    V = site_count(dims)
    seed = rank_seed(rank)
    with M.Chmc(dims, mag=0, beta=params["beta"], n_stout=0, seed=seed) as c:
        c.hot_start(seed)
        c.demon_microcanonical(args.warmup, params["e_max"], seed=seed)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        sampler = ClockSampler(gpu_index_for_smi()) if rank == 0 else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        torch.cuda.synchronize()
        res = c.demon_microcanonical(args.steps, params["e_max"], seed=seed + 1)
        torch.cuda.synchronize()
        dev_s = c.last_measure_ms() / 1e3  # CUDA events on the library's stream around the sweeps
        clocks = sampler.stop() if sampler else None
        # end to end: links in from pinned host memory, one sweep keeping them, links out
        Uh = torch.empty(V * 72, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(
            V, 4, 3, 3)
        c.get_gauge(out=Uh)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(args.steps):
            c.set_gauge(Uh)
            c.demon_microcanonical(1, params["e_max"], seed=seed + 2 + k, update_links=True)
            c.get_gauge(out=Uh)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    el = max_over_ranks(dev_s, dist, "cuda")
    wall = max_over_ranks(wall, dist, "cuda")
    if rank != 0:
        return
    sweep_s = el / args.steps
    flops = DEMON_FLOPS_PER_LINK * 4 * V / sweep_s / 1e12
    sm_peak = probe_fma_peak("fp64") / 148.0
    cpu = None
    if not args.no_cpu:
        import oracle as O

        U = O.gen_hot(dims, 1)
        t0 = time.perf_counter()
        O.demon_sweeps(dims, U, 1, 1, params["e_max"])
        tc = time.perf_counter() - t0
        cpu = {"value": 1.0 / tc, "unit": "sweeps/s", "cores": 1, "kind": "port",
               "sample": f"one sweep of the oracle over the {4 * V} links (sequential, one host thread)"}
    line = {
        "metric": DEMON_METRIC, "value": world / sweep_s, "unit": "sweeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sweep_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: Philox Haar hot start",
        "config": demon_config(args, params, world),
        "link_updates_per_s": world * 4 * V / sweep_s,
        "accepted": res["accepted"], "rejected": res["rejected"],
        "roofline": {"bound": "fp64 (one SM: the sweep is one CTA)", "achieved": flops, "peak": sm_peak,
                     "unit": "TFLOP/s", "frac": flops / sm_peak, "traffic": None,
                     "flops_per_link": DEMON_FLOPS_PER_LINK,
                     "peak_source": "measured CUDA-core FP64 FMA throughput / 148 SMs"},
        "cpu_baseline": cpu,
        "e2e": {"value": world * args.steps / wall, "unit": "sweeps/s", "h2d_bytes_per_step": 576 * V,
                "d2h_bytes_per_step": 576 * V + 48 + 8,
                "path": "mag_gauge_set + mag_demon_microcanonical (one sweep, links kept) + mag_gauge_get per step "
                        "from / to a pinned host buffer"},
        "clocks": clocks,
        "gpu_launches": 4 * args.steps,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    params = workload_params(args.workload)
    if args.impl == "reference":
        if params.get("kind") == "nersc":
            nersc_reference_arm(args, params, rank, world)
        elif params.get("kind") == "demon":
            demon_reference_arm(args, params, rank, world)
        elif params.get("kind") == "demon_ensemble":
            demon_ensemble_reference_arm(args, params, rank, world)
        else:
            reference_arm(args, params, rank, world)
        return
    if world > 1:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(world)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    torch.cuda.set_device(0)
    try:
        if params.get("kind") == "nersc":
            run_nersc(args, params, rank, world, dist)
        elif params.get("kind") == "demon":
            run_demon(args, params, rank, world, dist)
        elif params.get("kind") == "demon_ensemble":
            run_demon_ensemble(args, params, rank, world, dist)
        else:
            run_gpu(args, params, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
