"""Markov-chain parity on the GPU: whole runs of trajectories against the FP64 oracle.

* The FP64 GPU configuration at full size (16^3 x 32, Iwasaki beta = 2.25, three stout
  levels rho = 0.1, twelve force-gradient steps, mag = 2, Metropolis) for 20 trajectories
  against the oracle's records in tests/golden/run_16x16x16x32_3stout.json: H_old to 1e-12
  relative, Delta H to 1e-9 absolute, the same accept bit and the plaquette to 1e-12 on every
  trajectory.
* The 32^4 lattice of the mixed-versus-FP64 comparison (same action and smearing, sixteen
  force-gradient steps) for two trajectories against tests/golden/run_32x32x32x32_3stout.json,
  in FP64 at those bars and in mixed precision at the mixed ones (below).
* The 48^3 x 96 lattice of the Wilson-loop workload: Wilson loops, plaquettes and action sums
  of a hot start against tests/golden/hot_48x48x48x96_wloops.json.
* The mixed-precision path (FP32 staples, force and smearing on FP32 copies of the FP64
  master links; FP64 link integration, reunitarisation and Hamiltonian) from a thermalised
  6^4 configuration with three stout levels, against the oracle on the same momenta and
  uniforms:
    - single trajectories from one start: plaquette within 1e-7 of the oracle, Delta H
      within 5e-3, H_old to 1e-12 relative (the Hamiltonian is FP64 of the FP64 links);
    - a 12-trajectory Metropolis chain: the same accept/reject sequence as the oracle (with
      both outcomes present), the chain's mean plaquette within 1e-7 of the oracle's, mean
      Delta H and mean exp(-Delta H) within 1e-2;
    - reversibility (integrate, flip the momenta, integrate): max |U_back - U_0| below 1e-5
      and |H_back - H_0| below 5e-3 (FP64: 1e-10 and 1e-9).
* An ensemble of uneven chains (8^4 and 12^4, beta per chain, one stout level, eight
  force-gradient steps) in one context, every chain against its own oracle trajectory: FP64
  at the FP64 bars, mixed at the mixed ones.
"""
import json
import os

import numpy as np
import pytest

import mag_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _oracle_params(dims, **kw):
    return O.make_params(dims, mag=kw.get("mag", 2), action=1, beta=kw.get("beta", 2.25), c1=-0.331,
                         rho=kw.get("rho", 0.1), n_stout=kw.get("n_stout", 0), tau=kw.get("tau", 1.0),
                         n_steps=kw.get("n_steps", 8))


def _gpu_trajectory(c, U, P, u, chain_count=1):
    c.set_gauge(U)
    c.init_momentum(P)
    c.set_uniforms([u] * chain_count)
    (r,) = c.trajectory(refresh_momenta=False)
    return r


def _replay_records(name, precision):
    """Replays a fixture's run (same start, momenta and uniforms) on the GPU; returns
    (GPU records, oracle records)."""
    with open(os.path.join(GOLDEN, name)) as f:
        fx = json.load(f)
    dims = tuple(fx["dims"])
    p = fx["params"]
    seed = fx["rng_seed"]
    out = []
    with M.Chmc(dims, mag=p["mag"], action="iwasaki", beta=p["beta"], c1=p["c1"], rho=p["rho"],
                n_stout=p["n_stout"], tau=p["tau"], n_steps=p["n_steps"], precision=precision, seed=seed) as c:
        c.set_gauge(O.gen_hot(dims, fx["hot_seed"]))
        for t in range(len(fx["records"])):
            c.init_momentum(O.gen_momenta(dims, seed, t))
            c.set_uniforms([O.gen_uniform(seed, t)])
            (g,) = c.trajectory(refresh_momenta=False)
            out.append(g)
    return out, fx["records"]


def _check_fp64_records(recs, ref):
    """FP64 bars: H_old 1e-12 relative, the same accept bit, the plaquette to 1e-12, and Delta H
    to 1e-9 + 1e-11 |Delta H|.  The GPU and the oracle add the same terms in different orders, so
    their forces agree to rounding (the 1e-11 relative force bar) and a trajectory's energy
    change carries that relative difference: for |Delta H| <= 1 (equilibrium runs) the bar is
    1e-9 absolute; the first trajectories from a hot start change H by 10^2 (measured
    differences 3e-12 |Delta H| at 32^4)."""
    for t, (g, o) in enumerate(zip(recs, ref)):
        assert abs(g["h_old"] - o["h_old"]) <= 1e-12 * abs(o["h_old"]), t
        dh_tol = 1e-9 + 1e-11 * abs(o["delta_h"])
        assert abs(g["delta_h"] - o["delta_h"]) < dh_tol, (t, g["delta_h"], o["delta_h"])
        assert g["accept"] == o["accept"], t
        assert abs(g["avg_plaquette"] - o["avg_plaquette"]) < 1e-12, t


def test_config2_twenty_trajectories_against_the_oracle_records():
    recs, ref = _replay_records("run_16x16x16x32_3stout.json", "fp64")
    assert len(recs) == 20
    _check_fp64_records(recs, ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_32x32x32x32_trajectories_against_the_oracle_records(precision):
    """The lattice the mixed-versus-FP64 comparison is stated on, at full size, for the first two
    trajectories from a Haar hot start (Delta H -306 and -135): FP64 at the FP64 bars; mixed
    with the plaquette within 1e-7 of the oracle and the same accept bits (the mixed-precision
    bars), H_old to 1e-12 on the shared start, and Delta H within 5e-3 + 2e-3 |Delta H|.  The
    forces of a random start are far larger than at equilibrium, and their FP32 rounding moves
    Delta H by a fraction of its size (measured 1.0e-3 and 3.6e-4 of |Delta H|, plaquettes
    within 7.4e-10); at equilibrium the mixed-precision tests below hold Delta H to 5e-3."""
    recs, ref = _replay_records("run_32x32x32x32_3stout.json", precision)
    assert len(recs) == 2
    if precision == "fp64":
        _check_fp64_records(recs, ref)
        return
    diffs = [{"t": t, "h_old": g["h_old"] - o["h_old"], "delta_h": (g["delta_h"], o["delta_h"]),
              "plaquette": g["avg_plaquette"] - o["avg_plaquette"], "accept": (g["accept"], o["accept"])}
             for t, (g, o) in enumerate(zip(recs, ref))]
    for t, (g, o) in enumerate(zip(recs, ref)):
        h_tol = 1e-12 if t == 0 else 1e-7
        assert abs(g["h_old"] - o["h_old"]) <= h_tol * abs(o["h_old"]), diffs
        assert g["accept"] == o["accept"], diffs
        assert abs(g["avg_plaquette"] - o["avg_plaquette"]) < 1e-7, diffs
        assert abs(g["delta_h"] - o["delta_h"]) < 5e-3 + 2e-3 * abs(o["delta_h"]), diffs


def test_48x48x48x96_measurements_against_the_oracle_records():
    """The Wilson-loop workload's lattice at full size (48^3 x 96): a device hot start from
    Philox seed 6 (equal to the oracle's host-generated one to rounding) measured in the
    workload's context (mixed, three stout levels, beta 2.37; the measurements read the FP64
    master links) against the oracle: planar and off-axis Wilson loops, the average and the
    constrained plaquette to 1e-12; the thin plaquette and rectangle sums to 1e-12 relative."""
    with open(os.path.join(GOLDEN, "hot_48x48x48x96_wloops.json")) as f:
        fx = json.load(f)
    dims = tuple(fx["dims"])
    with M.Chmc(dims, mag=2, action="iwasaki", beta=2.37, c1=-0.331, rho=0.1, n_stout=3, n_steps=16,
                precision="mixed", seed=1) as c:
        c.hot_start(fx["hot_seed"])
        W = c.wilson_loops(8, 8)
        for e in fx["planar"]:
            assert abs(W[e["R"] - 1, e["T"] - 1] - e["w"]) < 1e-12, e
        for e in fx["off_axis"]:
            assert abs(c.avg_wilson_loop(e["r"], e["T"]) - e["w"]) < 1e-12, e
        assert abs(c.avg_plaquette() - fx["avg_plaquette"]) < 1e-12
        assert abs(c.check_constrained_plaquette() - fx["constrained_plaquette_mag2"]) < 1e-12
    with M.Chmc(dims, mag=2, action="iwasaki", beta=2.37, c1=-0.331, n_stout=0, precision="fp64", seed=1) as c:
        c.hot_start(fx["hot_seed"])
        plaq, rect, _ = c.gauge_action()
    assert abs(plaq - fx["plaq_sum"]) <= 1e-12 * abs(fx["plaq_sum"])
    assert abs(rect - fx["rect_sum"]) <= 1e-12 * abs(fx["rect_sum"])


DIMS6 = (6, 6, 6, 6)
KW6 = dict(mag=2, n_stout=3, rho=0.1, beta=2.25)


@pytest.fixture(scope="module")
def thermalised6():
    """A 6^4 configuration after 40 forced-accept FP64 trajectories from a Haar hot start
    (an input for the comparisons below: oracle and GPU both start from it)."""
    with M.Chmc(DIMS6, n_steps=6, precision="fp64", seed=91, n_forced_accept=40, **KW6) as c:
        c.hot_start(91)
        c.run_chmc(40)
        return c.get_gauge()


def test_mixed_single_trajectories_against_the_oracle(thermalised6):
    U0 = thermalised6
    po = _oracle_params(DIMS6, n_steps=12, **KW6)
    with M.Chmc(DIMS6, n_steps=12, precision="fp64", seed=7, **KW6) as c64, \
            M.Chmc(DIMS6, n_steps=12, precision="mixed", seed=7, **KW6) as c32:
        for k in range(4):
            P = O.gen_momenta(DIMS6, 7, 100 + k)
            _, o = O.trajectory(po, 100 + k, U0, P, 0.0, [0.0, 0.0])
            g64 = _gpu_trajectory(c64, U0, P, 0.0)
            g32 = _gpu_trajectory(c32, U0, P, 0.0)
            assert abs(g64["delta_h"] - o["delta_h"]) < 1e-9
            assert abs(g64["avg_plaquette"] - o["avg_plaquette"]) < 1e-12
            assert abs(g32["h_old"] - o["h_old"]) <= 1e-12 * abs(o["h_old"])
            assert abs(g32["avg_plaquette"] - o["avg_plaquette"]) < 1e-7, (k, g32["avg_plaquette"] - o["avg_plaquette"])
            assert abs(g32["delta_h"] - o["delta_h"]) < 5e-3, (k, g32["delta_h"], o["delta_h"])


def test_mixed_metropolis_chain_against_the_oracle(thermalised6):
    """12 Metropolis trajectories of 4 FG steps (large enough steps that both outcomes occur)."""
    n = 12
    po = _oracle_params(DIMS6, n_steps=4, **KW6)
    Uo = thermalised6.copy()
    demon = [0.0, 0.0]
    ro = []
    for t in range(n):
        P = O.gen_momenta(DIMS6, 8, 500 + t)
        Uo, o = O.trajectory(po, 500 + t, Uo, P, O.gen_uniform(8, 500 + t), demon)
        demon = o["demon"]
        ro.append(o)
    chains = {}
    for prec in ("fp64", "mixed"):
        with M.Chmc(DIMS6, n_steps=4, precision=prec, seed=8, **KW6) as c:
            c.set_gauge(thermalised6)
            rs = []
            for t in range(n):
                c.init_momentum(O.gen_momenta(DIMS6, 8, 500 + t))
                c.set_uniforms([O.gen_uniform(8, 500 + t)])
                (r,) = c.trajectory(refresh_momenta=False)
                rs.append(r)
            chains[prec] = rs
    acc_o = [o["accept"] for o in ro]
    assert 0 < sum(acc_o) < n, acc_o  # both outcomes occur
    for g, o in zip(chains["fp64"], ro):
        assert g["accept"] == o["accept"]
        assert abs(g["delta_h"] - o["delta_h"]) < 1e-9
        assert abs(g["avg_plaquette"] - o["avg_plaquette"]) < 1e-12
    m = chains["mixed"]
    assert [g["accept"] for g in m] == acc_o
    dh_o = np.array([o["delta_h"] for o in ro])
    dh_m = np.array([g["delta_h"] for g in m])
    pl_o = np.array([o["avg_plaquette"] for o in ro])
    pl_m = np.array([g["avg_plaquette"] for g in m])
    assert abs(pl_m.mean() - pl_o.mean()) < 1e-7, pl_m - pl_o
    assert abs(dh_m.mean() - dh_o.mean()) < 1e-2, dh_m - dh_o
    assert abs(np.exp(-dh_m).mean() - np.exp(-dh_o).mean()) < 1e-2


def test_mixed_reversibility(thermalised6):
    res = {}
    for prec in ("fp64", "mixed"):
        with M.Chmc(DIMS6, n_steps=12, precision=prec, seed=9, **KW6) as c:
            c.set_gauge(thermalised6)
            c.init_momentum(O.gen_momenta(DIMS6, 9, 0))
            H0, _ = c.get_hamiltonian()
            c.force_gradient_integrator()
            c.init_momentum(-c.get_momentum())
            c.force_gradient_integrator()
            H2, _ = c.get_hamiltonian()
            res[prec] = (np.abs(c.get_gauge() - thermalised6).max(), abs(H2 - H0))
    assert res["fp64"][0] < 1e-10 and res["fp64"][1] < 1e-9, res
    assert res["mixed"][0] < 1e-5 and res["mixed"][1] < 5e-3, res


ENS = [dict(dims=(8, 8, 8, 8), beta=2.1), dict(dims=(12, 12, 12, 12), beta=2.5), dict(dims=(8, 8, 8, 8), beta=2.35)]
ENS_KW = dict(mag=2, n_stout=1, rho=0.1, n_steps=8)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uneven_ensemble_chains_against_the_oracle(precision):
    n_traj = 2
    U = [O.gen_hot(ch["dims"], 50 + k) for k, ch in enumerate(ENS)]
    Uo = [u.copy() for u in U]
    with M.Chmc(chains=ENS, precision=precision, seed=60, **ENS_KW) as c:
        for k, u in enumerate(U):
            c.set_gauge(u, chain=k)
        for t in range(n_traj):
            Ps = [O.gen_momenta(ch["dims"], 60 + k, t) for k, ch in enumerate(ENS)]
            us = [O.gen_uniform(60 + k, t) for k in range(len(ENS))]
            for k, P in enumerate(Ps):
                c.init_momentum(P, chain=k)
            c.set_uniforms(us)
            recs = c.trajectory(refresh_momenta=False)
            for k, ch in enumerate(ENS):
                po = _oracle_params(ch["dims"], beta=ch["beta"], **ENS_KW)
                Uo[k], o = O.trajectory(po, t, Uo[k], Ps[k], us[k], [0.0, 0.0])
                g = recs[k]
                assert g["accept"] == o["accept"], (k, t)
                # mixed: from the second trajectory on the chain starts from links that differ from the
                # oracle's by the first trajectory's FP32 rounding (~1e-7), so H_old agrees to ~1e-8
                h_tol = 1e-12 if precision == "fp64" or t == 0 else 1e-7
                assert abs(g["h_old"] - o["h_old"]) <= h_tol * abs(o["h_old"]), (k, t)
                if precision == "fp64":
                    assert abs(g["delta_h"] - o["delta_h"]) < 1e-9, (k, t)
                    assert abs(g["avg_plaquette"] - o["avg_plaquette"]) < 1e-12, (k, t)
                    assert np.abs(c.get_gauge(k) - Uo[k]).max() < 1e-10, (k, t)
                else:
                    assert abs(g["delta_h"] - o["delta_h"]) < 5e-3, (k, t, g["delta_h"], o["delta_h"])
                    assert abs(g["avg_plaquette"] - o["avg_plaquette"]) < 1e-7, (k, t)
