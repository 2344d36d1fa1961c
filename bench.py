#!/usr/bin/env python
"""Benchmark of the B200 constrained SU(3) HMC path (one JSON line on rank 0).

A step is one HMC trajectory of the workload (momentum refresh, H_old, the
force-gradient molecular dynamics, reunitarisation, H_new, accept/reject),
replayed as one CUDA graph.  The default workload is the 16^3 x 32 lattice,
Iwasaki beta = 2.25 (c1 = -0.331), three stout levels rho = 0.1, twelve
force-gradient steps of tau = 1, constraint magnification 2, Metropolis accept,
plain FP64; the same lattice in mixed precision is measured beside it.

  python bench.py [--gpus N --steps K --warmup W] [--workload NAME] [--impl reference]

With --gpus N > 1 (launched by torchrun) every rank advances its own
independent chain on its own GPU: replicas, weak scaling, no collective in the
data path (the only collective is the max over ranks of the timing).

--impl reference times the reference's algorithm on the host cores: the
reference itself cannot be built here (it needs CPS, Qlattice, QMP, MPI), so
this is the FP64 CPU restatement in oracle/ (OpenMP over sites, as the
reference's field-hmc.h:385), run on a bounded sample and extrapolated.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HMC traj/s & force site-updates/s, mixed vs FP64 GPU at equal ΔH/plaquette"

WORKLOADS = {
    # 16^3 x 32, 3 stout levels, 12 FG steps, FP64 (the FP64 GPU path checked against the CPU oracle)
    "16x16x16x32_iwasaki_3stout": dict(dims=(16, 16, 16, 32), beta=2.25, n_stout=3, n_steps=12, precision="fp64"),
    # 32^4, 3 stout levels, 16 FG steps (mixed precision target beside FP64)
    "32x32x32x32_iwasaki_3stout": dict(dims=(32, 32, 32, 32), beta=2.25, n_stout=3, n_steps=16, precision="fp64"),
    # 8^4 thin-link Iwasaki, 8 FG steps (the CPU-runnable configuration)
    "8x8x8x8_iwasaki_thin": dict(dims=(8, 8, 8, 8), beta=2.25, n_stout=0, n_steps=8, precision="fp64"),
    # 48^3 x 96, beta 2.37, 3 stout levels, 16 FG steps
    "48x48x48x96_iwasaki_3stout": dict(dims=(48, 48, 48, 96), beta=2.37, n_stout=3, n_steps=16, precision="mixed"),
}
DEFAULT = "16x16x16x32_iwasaki_3stout"
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
    return ap.parse_args()


def workload_params(name: str) -> dict:
    p = dict(COMMON)
    p.update(WORKLOADS[name])
    return p


def site_count(dims) -> int:
    v = 1
    for d in dims:
        v *= d
    return v


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: str):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
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
        for line in open(self.path):
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
def cpu_sample(params: dict) -> dict:
    """Time the oracle (FP64, OpenMP) on one force evaluation, one link update
    and one Hamiltonian evaluation of the full workload; extrapolate to a
    trajectory: 4n forces + (4n+1) link updates + 2 Hamiltonians."""
    import numpy as np

    import oracle as O

    dims = params["dims"]
    po = O.make_params(dims, mag=params["mag"], action=1, beta=params["beta"], c1=params["c1"], rho=params["rho"],
                       n_stout=params["n_stout"], tau=params["tau"], n_steps=params["n_steps"])
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
    del np
    return {"t_force": t_force, "t_evolve": t_evolve, "t_ham": t_ham, "traj_s": traj_s,
            "cores": O.lib().mo_get_threads()}


def reference_arm(args, params, rank: int, world: int):
    if rank != 0:
        return
    import oracle as O

    dims = params["dims"]
    po = O.make_params(dims, mag=params["mag"], action=1, beta=params["beta"], c1=params["c1"], rho=params["rho"],
                       n_stout=params["n_stout"], tau=params["tau"], n_steps=params["n_steps"])
    U = O.gen_hot(dims, 1)
    P = O.gen_momenta(dims, 1, 0)
    t0 = time.perf_counter()
    O.evolve_gauge(po, U, P, 0.01)
    t_evolve = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.hamiltonian(po, U, P)
    t_ham = time.perf_counter() - t0
    for _ in range(args.warmup):
        O.force(po, U)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.force(po, U)
        ts.append(time.perf_counter() - t0)
    t_force = statistics.median(ts)
    n = params["n_steps"]
    traj_s = 4 * n * t_force + (4 * n + 1) * t_evolve + 2 * t_ham
    value = 1.0 / traj_s
    sample = (f"each step = one {params['n_stout']}-level stout Iwasaki force evaluation of the full lattice "
              f"(FP64 oracle port); trajectory = {4 * n} force evals + {4 * n + 1} link updates + 2 Hamiltonians")
    line = {
        "metric": METRIC, "value": value, "unit": "traj/s", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": traj_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: Philox Haar hot start",
        "config": config_of(args.workload, params, world),
        "cpu_baseline": {"value": value, "unit": "traj/s", "cores": O.lib().mo_get_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "force_evals_per_s": 1.0 / t_force,
        "site_updates_per_s": site_count(dims) / t_force,
    }
    print(json.dumps(line), flush=True)


def config_of(name, params, world):
    return {"workload": name, "lattice": "x".join(str(d) for d in params["dims"]), "action": "iwasaki",
            "beta": params["beta"], "c1": params["c1"], "stout_levels": params["n_stout"], "rho": params["rho"],
            "fg_steps": params["n_steps"], "tau": params["tau"], "mag": params["mag"],
            "precision": params["precision"], "accept": "metropolis", "parallelism": f"replicas{world}",
            "l2": "working set > 126 MB L2 (links, momenta, stout levels)"}


# ---------------------------------------------------------------- GPU arm
def run_gpu(args, params, rank, world, dist):
    import numpy as np
    import torch

    import mag_b200 as M
    from mag_b200.field_hmc import probe_fma_peak

    dims = params["dims"]
    V = site_count(dims)
    n = params["n_steps"]
    seed = 1000 + 7919 * rank
    kw = {k: v for k, v in params.items() if k != "dims"}

    def timed_run(prec: str):
        kk = dict(kw)
        kk["precision"] = prec
        kk["n_forced_accept"] = args.warmup  # the reference forces the first accepts (field-hmc.h:826)
        c = M.Chmc(dims, seed=seed, **kk)
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
        recs = c.run_chmc(args.steps)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        ms = c.last_run_ms()
        if dist:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return c, recs, ms, clocks

    c64, rec64, ms64, clocks = timed_run(params["precision"])
    head_prec = params["precision"]
    value = world * args.steps / (ms64 / 1e3)
    ms_per_step = ms64 / args.steps
    dh = [r[0]["delta_h"] for r in rec64]
    acc = [r[0]["accept"] for r in rec64]
    plaq = [r[0]["avg_plaquette"] for r in rec64]
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
    achieved = FLOPS_PER_SITE[dom] * V / (kt[dom] * 1e-3) / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        traffic = tj.get(f"{args.workload}:{head_prec}:{dom}")
    roofline = {"bound": prec_key, "kernel": dom, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic,
                "peak_source": f"measured CUDA-core {prec_key.upper()} FMA throughput (mag_probe_fma_peak)",
                "flops_per_site": FLOPS_PER_SITE[dom], "launch_ms": kt[dom],
                "kernel_ms": kt, "force_eval_ms": t_force_eval}
    # HBM roofline of the streaming link update
    ev_ms = c64.time_kernel("evolve", 5)
    bytes_evolve = V * 4 * (144 + 144 + 64)  # read U, write U, read P (FP64 master update)
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    roofline["evolve_hbm"] = {"achieved": bytes_evolve / (ev_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                              "frac": bytes_evolve / (ev_ms * 1e-3) / 1e9 / hbm_peak,
                              "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"}

    # end to end through the public API with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        field_bytes = V * 4 * 9 * 16
        Uh = torch.empty(V * 72, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(V, 4, 3, 3)
        Ph = torch.empty(V * 72, dtype=torch.float64, pin_memory=True).numpy().view(np.complex128).reshape(V, 4, 3, 3)
        Uh[:] = c64.get_gauge()
        rng = np.random.default_rng(seed)
        Ps = []
        for _ in range(args.e2e_steps):
            xi = rng.standard_normal((V, 4, 8))
            P = np.zeros((V, 4, 3, 3), np.complex128)
            s2, s6 = 1 / np.sqrt(2), 1 / np.sqrt(6)
            P[..., 0, 1] = (xi[..., 0] - 1j * xi[..., 1]) * s2
            P[..., 0, 2] = (xi[..., 3] - 1j * xi[..., 4]) * s2
            P[..., 1, 2] = (xi[..., 5] - 1j * xi[..., 6]) * s2
            P[..., 1, 0] = P[..., 0, 1].conj()
            P[..., 2, 0] = P[..., 0, 2].conj()
            P[..., 2, 1] = P[..., 1, 2].conj()
            P[..., 0, 0] = xi[..., 2] * s2 + xi[..., 7] * s6
            P[..., 1, 1] = -xi[..., 2] * s2 + xi[..., 7] * s6
            P[..., 2, 2] = -2 * xi[..., 7] * s6
            Ps.append(P)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(args.e2e_steps):
            c64.set_gauge(Uh)
            Ph[:] = Ps[k]
            c64.init_momentum(Ph)
            c64.set_uniforms([0.5])
            c64.trajectory(refresh_momenta=False)
            Uh[:] = c64.get_gauge()
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        if dist:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        e2e = {"value": world * args.e2e_steps / el, "unit": "traj/s", "h2d_bytes_per_step": 2 * field_bytes + 8,
               "d2h_bytes_per_step": field_bytes + 152, "steps": args.e2e_steps,
               "path": "mag_gauge_set + mag_momentum_set + mag_uniforms_set + mag_trajectory + mag_gauge_get"}
    c64.close()

    mixed = None
    if not args.no_mixed and head_prec == "fp64":
        cm, recm, msm, _ = timed_run("mixed")
        vm = world * args.steps / (msm / 1e3)
        mixed = {"value": vm, "unit": "traj/s", "ms_per_step": msm / args.steps, "speedup_vs_fp64": vm / value,
                 "delta_h_mean": statistics.fmean(r[0]["delta_h"] for r in recm),
                 "acceptance": statistics.fmean(r[0]["accept"] for r in recm),
                 "plaquette": recm[-1][0]["avg_plaquette"],
                 "force_eval_ms": cm.time_force(3)}
        cm.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        s = cpu_sample(params)
        cpu = {"value": 1.0 / s["traj_s"], "unit": "traj/s", "cores": s["cores"], "kind": "port",
               "sample": (f"oracle FP64 port, OpenMP: one force evaluation ({s['t_force']:.2f} s), one link update "
                          f"({s['t_evolve']:.2f} s) and one Hamiltonian ({s['t_ham']:.2f} s) of the full lattice, "
                          f"extrapolated to {4 * n} force evals + {4 * n + 1} updates + 2 Hamiltonians per trajectory"),
               "force_evals_per_s": 1.0 / s["t_force"]}

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "traj/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if head_prec == "fp64" else "f32+f64",
        "data": "synthetic: Philox Haar-random hot start, Gaussian momenta, Philox Metropolis uniforms",
        "config": config_of(args.workload, params, world),
        "force_evals_per_s": world * 4 * n * args.steps / (ms64 / 1e3),
        "site_updates_per_s": world * V * 4 * n * args.steps / (ms64 / 1e3),
        "delta_h_mean": statistics.fmean(dh), "delta_h_abs_mean": statistics.fmean(abs(x) for x in dh),
        "acceptance": statistics.fmean(acc), "plaquette": plaq[-1],
        "mixed": mixed, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
        "gpu_launches": kernels_per_traj * args.steps,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    params = workload_params(args.workload)
    if args.impl == "reference":
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
        run_gpu(args, params, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
