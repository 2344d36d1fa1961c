"""GPU parity: libmag_b200.so (sm_100a kernels, through the C ABI) against the
FP64 CPU oracle on the same seeded inputs.

Tolerances (plain FP64 GPU path): plaquette/action 1e-12 relative, per-link
force 1e-11 (relative to the largest force component), Delta H 1e-9
absolute, identical accept/reject and demon sequences.  Mixed precision
(FP32 staples/force/smearing on FP32 copies of FP64 master links): force 5e-5
relative; on the same trajectory as the FP64 path the same accept decision,
the plaquette within 1e-7 and Delta H within 5e-3 + 2e-3 |Delta H|.
"""
import numpy as np
import pytest

import mag_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu

DIMS = (4, 4, 4, 6)


def maxrel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def test_gauge_roundtrip_and_device_rng():
    with M.Chmc(DIMS, seed=21) as c:
        U = O.gen_hot(DIMS, 5)
        c.set_gauge(U)
        assert np.array_equal(c.get_gauge(), U)
        c.hot_start(5)
        assert np.abs(c.get_gauge() - U).max() < 1e-13
        c.init_momentum(None, traj=3)
        assert np.abs(c.get_momentum() - O.gen_momenta(DIMS, 21, 3)).max() < 1e-13
        P = O.gen_momenta(DIMS, 8, 0)
        c.init_momentum(P)
        assert np.abs(c.get_momentum() - P).max() < 1e-15


def _herm_traceless(rng, scale):
    A = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    H = (A + A.conj().T) / 2
    return (H - np.trace(H).real / 3 * np.eye(3)) * scale


def test_expiq_and_compute_lambda_match_the_oracle():
    """mag_expiq / mag_dexpiq / mag_compute_lambda (the reference's expiQ, DexpiQ and compute_Lambda
    for n matrices)
    against the oracle's literal restatement: Q of scale 0.01 to 2.5 (both signs of det Q, so the
    reflection branch too) and Q = 0 (the c1 = 0 branch)."""
    from mag_b200.field_hmc import compute_lambda, dexpiq, expiq

    rng = np.random.default_rng(5)
    n = 200
    Q = np.array([_herm_traceless(rng, (0.01, 0.1, 1.0, 2.5)[i % 4]) for i in range(n)])
    Q[0] = 0.0
    S = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    U = O.gen_hot((2, 2, 4, 4), 3).reshape(-1, 3, 3)[:n]
    E = expiq(Q)
    Eo = np.array([O.expiQ(q) for q in Q])
    assert np.array_equal(E[0], np.eye(3))
    dE = np.abs(E - Eo).max()
    L = compute_lambda(Q, S, U)
    Lo = np.array([O.compute_lambda(q, s, u) for q, s, u in zip(Q, S, U)])
    assert np.all(L[0] == 0)
    dL = max(np.abs(L[i] - Lo[i]).max() / max(1.0, np.abs(Lo[i]).max()) for i in range(n))
    assert dE < 1e-14
    assert dL < 1e-12
    D = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    G = dexpiq(Q, D)
    Go = np.array([O.dexpiQ(q, d) for q, d in zip(Q, D)])
    assert np.all(G[0] == 0)
    dG = max(np.abs(G[i] - Go[i]).max() / max(1.0, np.abs(Go[i]).max()) for i in range(n))
    assert dG < 1e-12
    assert sum(1 for q in Q if np.linalg.det(q).real < 0) > 10  # the reflection branch is exercised


def test_kinetic_energy_and_trajectory_counter():
    """The kinetic part of get_hamiltonian (constrained last links excluded) and the trajectory
    counter that selects each trajectory's Philox momenta and uniform."""
    po = O.make_params(DIMS, mag=2, action=1, beta=2.25, n_stout=0, n_steps=8)
    U = O.gen_hot(DIMS, 9)
    with M.Chmc(DIMS, mag=2, seed=21) as c:
        c.set_gauge(U)
        P = O.gen_momenta(DIMS, 3, 1)
        c.init_momentum(P)
        ko = O.kinetic(po, P)
        assert abs(c.kinetic_energy() - ko) <= 1e-12 * abs(ko)
        assert c.traj_counter() == 0
        c.set_traj_counter(5)
        assert c.traj_counter() == 5
        (rec,) = c.trajectory()
        assert c.traj_counter() == 6
        k5 = O.kinetic(po, O.gen_momenta(DIMS, 21, 5))
        assert abs(rec["kinetic_old"] - k5) <= 1e-12 * abs(k5)
        assert rec["uniform"] == O.gen_uniform(21, 5)


@pytest.mark.parametrize("action,mag,n_stout", [
    ("iwasaki", 0, 0), ("wilson", 0, 0), ("iwasaki", 2, 0), ("wilson", 2, 0),
    ("iwasaki", 0, 1), ("iwasaki", 0, 3), ("iwasaki", 2, 3), ("wilson", 2, 1)])
def test_force_parity_fp64(action, mag, n_stout):
    U = O.gen_hot(DIMS, 7)
    po = O.make_params(DIMS, mag=mag, action=1 if action == "iwasaki" else 0, n_stout=n_stout, rho=0.1)
    with M.Chmc(DIMS, mag=mag, action=action, n_stout=n_stout, rho=0.1) as c:
        c.set_gauge(U)
        F = c.get_force()
    Fo = O.force(po, U)
    assert maxrel(F, Fo) < 1e-11


@pytest.mark.parametrize("action", ["iwasaki", "wilson"])
def test_staple_and_action_parity(action):
    U = O.gen_hot(DIMS, 9)
    a = 1 if action == "iwasaki" else 0
    po = O.make_params(DIMS, action=a)
    with M.Chmc(DIMS, action=action, mag=0) as c:
        c.set_gauge(U)
        V = c.get_extended_staple_dagger()
        p, r, s = c.gauge_action()
        avg = c.avg_plaquette()
    assert maxrel(V, O.staple_dagger(po, U)) < 1e-12
    po_, ro_, so_ = O.action(po, U)
    assert abs(p - po_) <= 1e-12 * abs(po_) + 1e-12
    assert abs(r - ro_) <= 1e-12 * abs(ro_) + 1e-12
    assert abs(s - so_) <= 1e-12 * abs(so_)
    assert abs(avg - O.avg_plaquette(DIMS, U)) < 1e-14


def test_smeared_action_and_levels_parity():
    U = O.gen_hot(DIMS, 10)
    po = O.make_params(DIMS, n_stout=3, rho=0.1)
    lv = O.stout_forward(po, U)
    with M.Chmc(DIMS, n_stout=3, rho=0.1) as c:
        c.set_gauge(U)
        for k in range(4):
            assert np.abs(c.stout_level(k) - lv[k]).max() < 1e-13
        p, r, s = c.gauge_action()
    po_, ro_, so_ = O.action(po, U)
    assert abs(s - so_) <= 1e-12 * abs(so_)
    assert abs(p - po_) <= 1e-12 * abs(po_)


@pytest.mark.parametrize("mag", [0, 2])
def test_hamiltonian_and_updates_parity(mag):
    U = O.gen_hot(DIMS, 11)
    P = O.gen_momenta(DIMS, 3, 0)
    po = O.make_params(DIMS, mag=mag)
    with M.Chmc(DIMS, mag=mag) as c:
        c.set_gauge(U)
        c.init_momentum(P)
        H, parts = c.get_hamiltonian()
        ho = O.hamiltonian(po, U, P)
        assert abs(H - ho["H"]) <= 1e-12 * abs(ho["H"])
        assert abs(parts[0] - ho["kinetic"]) <= 1e-12 * abs(ho["kinetic"])
        c.evolve_gauge_field(0.1)
        U1 = O.evolve_gauge(po, U, P, 0.1)
        assert np.abs(c.get_gauge() - U1).max() < 1e-13
        c.evolve_momentum(0.05)
        P1 = O.evolve_momentum(DIMS, P, O.force(po, U1), 0.05)
        assert np.abs(c.get_momentum() - P1).max() < 1e-11


def test_reunitarize_parity():
    U = O.gen_hot(DIMS, 12)
    rng = np.random.default_rng(0)
    Un = U + 1e-6 * (rng.normal(size=U.shape) + 1j * rng.normal(size=U.shape))
    with M.Chmc(DIMS) as c:
        c.set_gauge(Un)
        (dev,) = c.reunitarize()
        Ug = c.get_gauge()
    Uo, devo = O.reunitarize(DIMS, Un)
    assert np.abs(Ug - Uo).max() < 1e-15
    assert abs(dev - devo) < 1e-15


def _run_pair(dims, kw, n_traj, seed=31, start_seed=4):
    """Trajectories on GPU (host momenta/uniforms) and oracle; returns records."""
    po = O.make_params(dims, mag=kw.get("mag", 2), action=1 if kw.get("action", "iwasaki") == "iwasaki" else 0,
                       beta=kw.get("beta", 2.25), n_stout=kw.get("n_stout", 0), rho=kw.get("rho", 0.1),
                       n_steps=kw.get("n_steps", 8), tau=kw.get("tau", 1.0),
                       accept=1 if kw.get("accept", "metropolis") == "demon" else 0, e_max=kw.get("e_max", 100.0),
                       integrator=1 if kw.get("integrator", "fg") == "leapfrog" else 0,
                       n_forced=kw.get("n_forced_accept", 0))
    U = O.gen_hot(dims, start_seed)
    Uo = U.copy()
    demon = [0.0, 0.0]
    out = []
    with M.Chmc(dims, seed=seed, **kw) as c:
        c.set_gauge(U)
        for t in range(n_traj):
            P = O.gen_momenta(dims, seed, t)
            u = O.gen_uniform(seed, t)
            c.init_momentum(P)
            c.set_uniforms([u])
            (g,) = c.trajectory(refresh_momenta=False)
            Uo, o = O.trajectory(po, t, Uo, P, u, demon)
            demon = o["demon"]
            out.append((g, o, np.abs(c.get_gauge() - Uo).max()))
    return out


def test_trajectory_parity_8x4_iwasaki_fp64_metropolis():
    # the CPU-runnable configuration: 8^4, Iwasaki beta = 2.25, 8 force-gradient steps
    res = _run_pair((8, 8, 8, 8), dict(mag=2, n_steps=8), 3)
    for g, o, du in res:
        assert abs(g["h_old"] - o["h_old"]) <= 1e-12 * abs(o["h_old"])
        assert abs(g["delta_h"] - o["delta_h"]) < 1e-9
        assert g["accept"] == o["accept"]
        assert abs(g["avg_plaquette"] - o["avg_plaquette"]) < 1e-12
        assert du < 1e-10


def test_forced_accepts_then_metropolis():
    """num_forced_accept_step (field-hmc.h:826): the first trajectories are accepted whatever
    Delta H; with 2 coarse steps trajectory 1 has Delta H ~ 1e2 and is kept only because it is
    forced, trajectories 2 and 3 fall back to Metropolis."""
    res = _run_pair((4, 4, 4, 4), dict(mag=2, n_steps=2, n_forced_accept=2), 4)
    assert [g["accept"] for g, _, _ in res][:2] == [1, 1]
    assert res[1][1]["delta_h"] > 10.0
    for g, o, du in res:
        assert g["accept"] == o["accept"]
        assert abs(g["delta_h"] - o["delta_h"]) < 1e-9
        assert du < 1e-10


def test_trajectory_parity_half_length_trajectory():
    # tau = 0.5 with 4 force-gradient steps (dt = tau / n_steps), one stout level
    res = _run_pair((4, 4, 4, 6), dict(mag=2, n_steps=4, tau=0.5, n_stout=1), 2)
    for g, o, du in res:
        assert abs(g["delta_h"] - o["delta_h"]) < 1e-9
        assert g["accept"] == o["accept"]
        assert du < 1e-10


def test_trajectory_parity_demon_sequence():
    res = _run_pair((8, 8, 8, 8), dict(mag=2, n_steps=8, accept="demon", e_max=60.0), 3)
    for g, o, _ in res:
        assert g["accept"] == o["accept"]
        assert abs(g["demon"][0] - o["demon"][0]) < 1e-8
        assert abs(g["demon"][1] - o["demon"][1]) < 1e-8


def test_trajectory_parity_three_stout_levels():
    res = _run_pair((4, 4, 4, 8), dict(mag=2, n_stout=3, rho=0.1, n_steps=12), 2)
    for g, o, du in res:
        assert abs(g["delta_h"] - o["delta_h"]) < 1e-9
        assert g["accept"] == o["accept"]
        assert du < 1e-10


@pytest.mark.slow
def test_trajectory_parity_16x16x16x32_three_stout_full_size():
    """The FP64 GPU configuration at its full size: 16^3 x 32, Iwasaki beta = 2.25, three
    stout levels rho = 0.1, twelve force-gradient steps, one trajectory against the oracle
    (about 100 s of oracle time on 16 host threads)."""
    res = _run_pair((16, 16, 16, 32), dict(mag=2, n_stout=3, rho=0.1, n_steps=12), 1)
    g, o, du = res[0]
    assert abs(g["h_old"] - o["h_old"]) <= 1e-12 * abs(o["h_old"])
    assert abs(g["delta_h"] - o["delta_h"]) < 1e-9
    assert g["accept"] == o["accept"]
    assert abs(g["avg_plaquette"] - o["avg_plaquette"]) < 1e-12
    assert du < 1e-10


def test_leapfrog_parity():
    res = _run_pair((4, 4, 4, 4), dict(mag=0, n_steps=6, integrator="leapfrog"), 1)
    g, o, du = res[0]
    assert abs(g["delta_h"] - o["delta_h"]) < 1e-9 and du < 1e-10


def test_graph_run_matches_eager_trajectories():
    dims = (4, 4, 4, 8)
    with M.Chmc(dims, seed=41, n_stout=1, n_steps=4) as a, M.Chmc(dims, seed=41, n_stout=1, n_steps=4) as b:
        a.hot_start(2)
        b.hot_start(2)
        ra = a.run_chmc(3)
        rb = [b.trajectory(True) for _ in range(3)]
        for x, y in zip(ra, rb):
            assert x[0]["delta_h"] == y[0]["delta_h"] and x[0]["accept"] == y[0]["accept"]
        assert np.array_equal(a.get_gauge(), b.get_gauge())


def test_ensemble_chains_equal_single_lattices():
    chains = [dict(dims=(4, 4, 4, 4), beta=2.0), dict(dims=(4, 4, 6, 6), beta=2.3), dict(dims=(6, 6, 6, 6), beta=2.6)]
    common = dict(mag=2, n_stout=1, rho=0.1, n_steps=4, seed=100)
    with M.Chmc(chains=chains, **common) as e:
        e.hot_start(9)
        re = e.run_chmc(2)
        Ue = [e.get_gauge(k) for k in range(3)]
    for k, ch in enumerate(chains):
        kw = dict(common)
        kw["seed"] = 100 + k
        with M.Chmc(ch["dims"], beta=ch["beta"], **kw) as s:
            # chain k of the ensemble draws its hot start from seed + k
            s.hot_start(9 + k)
            rs = s.run_chmc(2)
            assert np.array_equal(s.get_gauge(), Ue[k])
        for t in range(2):
            assert re[t][k]["delta_h"] == rs[t][0]["delta_h"]


def test_wilson_loops_parity():
    U = O.gen_hot(DIMS, 14)
    with M.Chmc(DIMS) as c:
        c.set_gauge(U)
        W = c.wilson_loops(3, 4)
        for R in range(1, 4):
            for T in range(1, 5):
                assert abs(W[R - 1, T - 1] - O.wilson_loop(DIMS, U, (R, 0, 0), T)) < 1e-13
        assert abs(c.avg_wilson_loop((1, 2, 0), 2) - O.wilson_loop(DIMS, U, (1, 2, 0), 2)) < 1e-13
        for r, T in (((1, 1, 1), 2), ((2, 1, 1), 3)):  # spatial displacements along all three directions
            assert abs(c.avg_wilson_loop(r, T) - O.wilson_loop(DIMS, U, r, T)) < 1e-13
        c.cold_start()
        assert np.abs(c.wilson_loops(2, 2) - 3.0).max() < 1e-14


def test_constrained_plaquette_parity_and_invariance():
    U = O.gen_hot((4, 4, 4, 4), 15)
    with M.Chmc((4, 4, 4, 4), mag=2, n_steps=4, seed=3) as c:
        c.set_gauge(U)
        cp = c.check_constrained_plaquette()
        assert abs(cp - O.constrained_plaquette((4, 4, 4, 4), U, 2)) < 1e-14
        c.init_momentum(None, traj=0)
        c.force_gradient_integrator()
        assert abs(c.check_constrained_plaquette() - cp) < 1e-12


def test_reversibility_fp64():
    dims = (4, 4, 4, 8)
    with M.Chmc(dims, mag=2, n_stout=2, n_steps=6) as c:
        c.hot_start(3)
        U0 = c.get_gauge()
        c.init_momentum(None, traj=0)
        P0 = c.get_momentum()
        c.force_gradient_integrator()
        c.init_momentum(-c.get_momentum())
        c.force_gradient_integrator()
        assert np.abs(c.get_gauge() - U0).max() < 1e-10
        assert np.abs(c.get_momentum() + P0).max() < 1e-9


def test_mixed_precision_force_and_trajectory():
    dims = (4, 4, 4, 8)
    U = O.gen_hot(dims, 16)
    po = O.make_params(dims, mag=2, n_stout=3, rho=0.1)
    with M.Chmc(dims, mag=2, n_stout=3, rho=0.1, precision="mixed") as c:
        c.set_gauge(U)
        assert maxrel(c.get_force(), O.force(po, U)) < 5e-5
    r = {}
    for prec in ("fp64", "mixed"):
        with M.Chmc(dims, mag=2, n_stout=3, rho=0.1, n_steps=12, precision=prec, seed=5) as c:
            c.set_gauge(U)
            (r[prec],) = c.trajectory(True)
    # the Hamiltonian is FP64 of the FP64 master links in both paths; the mixed MD moves the
    # links by FP32 forces: the same accept decision, the plaquette within 1e-7, and Delta H
    # within the FP32 force rounding of a hot start (5e-3 + 2e-3 |Delta H|)
    assert abs(r["mixed"]["h_old"] - r["fp64"]["h_old"]) <= 1e-12 * abs(r["fp64"]["h_old"])
    assert r["mixed"]["accept"] == r["fp64"]["accept"]
    assert abs(r["mixed"]["delta_h"] - r["fp64"]["delta_h"]) < 5e-3 + 2e-3 * abs(r["fp64"]["delta_h"])
    assert abs(r["mixed"]["avg_plaquette"] - r["fp64"]["avg_plaquette"]) < 1e-7


def test_nan_is_reported_as_error_status():
    U = O.gen_hot((4, 4, 4, 4), 17)
    U[3, 1, 0, 0] = np.nan
    with M.Chmc((4, 4, 4, 4), n_steps=2) as c:
        c.set_gauge(U)
        with pytest.raises(M.MagError) as e:
            c.trajectory(True)
        assert e.value.code == -3


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_evolve_by_force_matches_oracle(precision):
    """U <- exp(i dt F(U)) U (the force-gradient link update) against the oracle's
    evolve_gauge driven by its own force; constrained Iwasaki with one stout level."""
    U = O.gen_hot(DIMS, 31)
    po = O.make_params(DIMS, mag=2, action=1, n_stout=1, rho=0.1)
    with M.Chmc(DIMS, mag=2, action="iwasaki", n_stout=1, rho=0.1, precision=precision) as c:
        c.set_gauge(U)
        c.evolve_gauge_field(0.05, src="force")
        Ug = c.get_gauge()
    Uo = O.evolve_gauge(po, U, O.force(po, U), 0.05)
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert np.abs(Ug - Uo).max() < tol


def test_alias_entry_points():
    """mag_stout_forward / mag_stout_force / mag_fg_trajectory / mag_batch_* are the same calls."""
    import ctypes

    from mag_b200 import _lib

    L = _lib.load()
    U = O.gen_hot(DIMS, 32)
    with M.Chmc(DIMS, n_stout=2, rho=0.1, seed=4) as c:
        c.set_gauge(U)
        a = np.zeros_like(U)
        _lib.check(L.mag_stout_forward(c._h, 0, 2, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "sf")
        assert np.array_equal(a, c.stout_level(2))
        f = np.zeros_like(U)
        _lib.check(L.mag_stout_force(c._h, 0, f.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "sF")
        assert np.array_equal(f, c.get_force())
        r = _lib.TrajResult()
        _lib.check(L.mag_fg_trajectory(c._h, 1, ctypes.byref(r)), "fg")
        assert np.isfinite(r.delta_h)
    with M.Chmc(DIMS, n_stout=0) as c:
        code = L.mag_stout_force(c._h, 0, np.zeros((O.volume(DIMS), 4, 3, 3), np.complex128).ctypes.data_as(
            ctypes.POINTER(ctypes.c_double)))
        assert code == _lib.MAG_ERR_STATE
    # mag_batch_create / mag_batch_run against mag_ensemble_create / mag_run: identical records
    from mag_b200.field_hmc import make_params

    plist = [make_params((4, 4, 4, 4), n_stout=1, seed=6), make_params((4, 4, 4, 6), n_stout=1, beta=2.4, seed=6)]
    arr = (_lib.MagParams * 2)(*plist)
    recs = []
    for create, run in ((L.mag_batch_create, L.mag_batch_run), (L.mag_ensemble_create, L.mag_run)):
        h = ctypes.c_void_p()
        _lib.check(create(arr, 2, ctypes.byref(h)), "create")
        try:
            _lib.check(L.mag_gauge_hot_start(h, 3), "hot start")
            res = (_lib.TrajResult * 4)()
            _lib.check(run(h, 2, res), "run")
            recs.append([(r.delta_h, r.accept, r.h_old) for r in res])
        finally:
            L.mag_ctx_destroy(h)
    assert recs[0] == recs[1] and all(np.isfinite(d) for d, _, _ in recs[0])


def test_split_ensemble_reproduces_the_single_context():
    """Chains 0-3 in one context, or chains {0, 3} and {1, 2} in two contexts with their
    ensemble stream indices: identical per-chain trajectories (bit for bit)."""
    chains = [dict(dims=(4, 4, 4, 4), beta=2.1), dict(dims=(4, 4, 4, 6), beta=2.3),
              dict(dims=(4, 4, 4, 4), beta=2.4), dict(dims=(4, 4, 6, 6), beta=2.2)]
    kw = dict(n_stout=1, rho=0.1, n_steps=4, seed=17)
    with M.Chmc(chains=chains, **kw) as c:
        c.hot_start(17)
        whole = c.run_chmc(3)
        U_whole = [c.get_gauge(k) for k in range(4)]
    for part in ([0, 3], [1, 2]):
        with M.Chmc(chains=[chains[i] for i in part], **kw) as c:
            c.set_stream_index(part)
            c.hot_start(17)
            rec = c.run_chmc(3)
            for j, i in enumerate(part):
                for t in range(3):
                    assert rec[t][j]["delta_h"] == whole[t][i]["delta_h"]
                    assert rec[t][j]["accept"] == whole[t][i]["accept"]
                assert np.array_equal(c.get_gauge(j), U_whole[i])


@pytest.mark.parametrize("dims,mag,n_stout", [((2, 2, 4, 4), 2, 0), ((2, 4, 2, 6), 2, 1), ((8, 4, 4, 8), 4, 0),
                                             ((8, 4, 4, 8), 4, 2), ((6, 2, 10, 4), 0, 1)])
def test_edge_lattices_force_action_and_trajectory(dims, mag, n_stout):
    """Extents of 2 (rectangles wrap onto themselves), odd multiples, mag = 4 segments and no
    constraint: force, action and one trajectory against the oracle."""
    U = O.gen_hot(dims, 13)
    po = O.make_params(dims, mag=mag, action=1, n_stout=n_stout, rho=0.1, n_steps=4)
    with M.Chmc(dims, mag=mag, n_stout=n_stout, rho=0.1, n_steps=4, seed=2) as c:
        c.set_gauge(U)
        assert maxrel(c.get_force(), O.force(po, U)) < 1e-11
        p, r, a = c.gauge_action()
        pa, ra, aa = O.action(po, U)
        assert abs(p - pa) <= 1e-12 * abs(pa) and abs(r - ra) <= 1e-12 * abs(ra) and abs(a - aa) <= 1e-12 * abs(aa)
    res = _run_pair(dims, dict(mag=mag, n_stout=n_stout, rho=0.1, n_steps=4), 1, start_seed=13)
    g, o, du = res[0]
    assert abs(g["delta_h"] - o["delta_h"]) < 1e-9 and g["accept"] == o["accept"] and du < 1e-10


@pytest.mark.parametrize("n_stout,mag,pair", [(3, 0, False), (3, 2, True), (1, 2, False)])
def test_gpu_force_is_minus_gpu_action_derivative(n_stout, mag, pair):
    """The stout chain rule on the GPU against a central finite difference of the GPU's own
    smeared action: -Re Tr(X F(x,mu)) = dS/deps for U(x,mu) -> exp(i eps X) U(x,mu), or for a
    constrained pair U(x,mu) -> U(x,mu) exp(-i eps X), U(x+mu,mu) -> exp(i eps X) U(x+mu,mu)."""
    dims = (4, 4, 4, 6)
    U = O.gen_hot(dims, 21)
    rng = np.random.default_rng(5)
    X = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    X = X + X.conj().T
    X -= np.trace(X) / 3 * np.eye(3)
    # a pair: (0,0,0,0) along mu = 1, the first link of its mag = 2 segment, and (0,1,0,0);
    # a single link: (1,0,0,0) along mu = 1, a free link (x0 odd)
    mu = 1
    site = 0 if pair else 1
    nxt = dims[0]
    with M.Chmc(dims, mag=mag, n_stout=n_stout, rho=0.1) as c:
        c.set_gauge(U)
        F = c.get_force()

        def S(eps):
            V = U.copy()
            if pair:
                V[site, mu] = V[site, mu] @ O.expiQ(-X * eps)
                V[nxt, mu] = O.expiQ(X * eps) @ V[nxt, mu]
            else:
                V[site, mu] = O.expiQ(X * eps) @ V[site, mu]
            c.set_gauge(V)
            return c.gauge_action()[2]

        h = 1e-5
        fd = (S(h) - S(-h)) / (2 * h)
    # the pair moves along the segment; its derivative is the force of the segment's first link
    an = -np.trace(X @ F[site, mu]).real
    assert abs(fd - an) < 2e-7 * max(1.0, abs(an)), (fd, an)



VARIANTS = ["t1m2", "t1m3", "t1m4", "t1m5", "s3r168", "s3r128", "s6r168", "s6r128", "s6r96"]


@pytest.mark.parametrize("dims,action,mag,n_stout,family", [
    ((4, 4, 4, 6), "iwasaki", 2, 0, "force"), ((5, 3, 3, 4), "wilson", 0, 0, "force"),
    ((4, 4, 4, 6), "iwasaki", 2, 3, "staple"), ((4, 4, 4, 6), "iwasaki", 2, 3, "stout_chain"),
    ((5, 3, 3, 4), "iwasaki", 0, 1, "staple"), ((5, 3, 3, 4), "iwasaki", 0, 1, "stout_chain")])
def test_every_kernel_variant_matches_the_oracle(dims, action, mag, n_stout, family):
    """Each launch shape of the tuner (one thread per link at four register caps; the direction
    split with 3 or 6 warps per 32-link tile at three caps) gives the force the oracle gives:
    FP64 to 1e-11, FP32 (mixed) to 5e-5; 5 x 3 x 3 x 4 has a partial last tile."""
    U = O.gen_hot(dims, 19)
    po = O.make_params(dims, mag=mag, action=1 if action == "iwasaki" else 0, n_stout=n_stout, rho=0.1)
    Fo = O.force(po, U)
    for prec, tol in (("fp64", 1e-11), ("mixed", 5e-5)):
        with M.Chmc(dims, mag=mag, action=action, n_stout=n_stout, rho=0.1, precision=prec) as c:
            c.set_gauge(U)
            for v in VARIANTS:
                c.set_kernel_variant(family, "fp64" if prec == "fp64" else "fp32", v)
                assert maxrel(c.get_force(), Fo) < tol, (prec, v)


def test_fma_throughput_probes():
    """mag_probe_fma_peak: every mode measures a finite throughput, FP32 above FP64; others are refused."""
    import ctypes

    from mag_b200 import _lib
    from mag_b200.field_hmc import probe_fma_peak

    r = {p: probe_fma_peak(p) for p in ("fp64", "fp32", "fp32x2", "fp32x2_selected")}
    assert all(np.isfinite(v) and v > 1.0 for v in r.values()), r
    assert r["fp32"] > r["fp64"], r
    v = ctypes.c_double()
    assert _lib.load().mag_probe_fma_peak(4, ctypes.byref(v)) != 0
