"""CPU tests of the FP64 oracle: known answers and invariants.

The reference ships no golden vectors, so the oracle is pinned by
  * published known-answer vectors of Philox-4x32-10 (Random123 kat_vectors),
  * exact results (unit links, the reference's own Taylor exp at field-hmc.h:73-80),
  * invariants: unitarity, gauge invariance, force = -dS/dU by central finite
    differences, force-gradient / leapfrog order, reversibility, invariance of
    the constrained plaquette (quench_test/main.C:115-145).
"""
import numpy as np
import pytest

import oracle as O

DIMS = (4, 4, 4, 6)


def rand_herm(rng, scale=1.0):
    X = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    X = X + X.conj().T
    X -= np.trace(X) / 3 * np.eye(3)
    return X * scale


def idx(dims, x):
    return x[0] + dims[0] * (x[1] + dims[1] * (x[2] + dims[2] * x[3]))


# ------------------------------------------------------------------ RNG
def test_philox_known_answers():
    # Random123 kat_vectors, philox4x32_10
    assert O.philox4x32([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox4x32([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox4x32([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_momenta_are_hermitian_traceless_unit_gaussians():
    P = O.gen_momenta((4, 4, 4, 4), 11, 0)
    assert np.abs(P - P.conj().transpose(0, 1, 3, 2)).max() < 1e-15
    assert np.abs(np.trace(P, axis1=2, axis2=3)).max() < 1e-14
    # Tr(P^2) = sum_a xi_a^2 with xi ~ N(0, 1): mean 8 per link
    t = np.einsum("slij,slji->sl", P, P).real
    assert abs(t.mean() - 8.0) < 0.25
    # different trajectories and seeds give different momenta
    assert np.abs(P - O.gen_momenta((4, 4, 4, 4), 11, 1)).max() > 0.1
    assert np.abs(P - O.gen_momenta((4, 4, 4, 4), 12, 0)).max() > 0.1


def test_uniforms_in_unit_interval():
    u = [O.gen_uniform(5, t) for t in range(200)]
    assert min(u) > 0.0 and max(u) < 1.0
    assert abs(np.mean(u) - 0.5) < 0.08


def test_hot_start_is_special_unitary():
    U = O.gen_hot(DIMS, 3)
    I = np.eye(3)
    assert np.abs(np.einsum("slij,slkj->slik", U, U.conj()) - I).max() < 1e-14
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-14


# ------------------------------------------------------------------ SU(3) algebra
def test_expiQ_matches_taylor_series():
    rng = np.random.default_rng(0)
    for scale in (1e-3, 0.05, 0.3, 1.0):
        Q = rand_herm(rng, scale)
        # the reference's alternative exp (field-hmc.h:73-80) is a truncated Taylor
        # series; use enough terms to be exact in double
        iQ = 1j * Q
        E, term = np.eye(3, dtype=complex), np.eye(3, dtype=complex)
        for k in range(1, 40):
            term = term @ iQ / k
            E = E + term
        assert np.abs(O.expiQ(Q) - E).max() < 1e-13
    assert np.abs(O.expiQ(np.zeros((3, 3))) - np.eye(3)).max() == 0.0


def test_expiQ_negative_c0_branch():
    # c0 < 0 takes the reflection branch of field-hmc.h:90-93 and 111-115
    Q = np.diag([-0.9, 0.2, 0.7]).astype(complex)
    assert np.trace(Q @ Q @ Q).real < 0
    assert np.abs(O.expiQ(Q) - np.diag(np.exp(1j * np.diag(Q)))).max() < 1e-14


def test_dexpiQ_is_the_derivative_of_expiQ():
    rng = np.random.default_rng(1)
    for scale in (0.02, 0.4, 1.5):
        Q = rand_herm(rng, scale)
        D = rand_herm(rng, 1.0)
        h = 1e-6
        fd = (O.expiQ(Q + h * D) - O.expiQ(Q - h * D)) / (2 * h)
        assert np.abs(O.dexpiQ(Q, D) - fd).max() < 1e-8


def test_compute_lambda_contracts_the_derivative():
    # Re Tr(d e^{iQ} U S') = Tr(dQ Lambda)  (hep-lat/0311018 eq. 72-74)
    rng = np.random.default_rng(2)
    Q = rand_herm(rng, 0.3)
    U = O.gen_hot((1, 1, 1, 1), 9)[0, 0]
    S = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    lam = O.compute_lambda(Q, S, U)
    assert np.abs(lam - lam.conj().T).max() < 1e-14
    assert abs(np.trace(lam)) < 1e-14
    for _ in range(3):
        D = rand_herm(rng)
        lhs = np.trace(O.dexpiQ(Q, D) @ U @ S).real
        rhs = np.trace(D @ lam).real
        assert abs(lhs - rhs) < 1e-12 * max(1.0, abs(lhs))


def test_unitarize_projects_onto_su3():
    rng = np.random.default_rng(3)
    U = O.gen_hot((1, 1, 1, 1), 4)[0, 0]
    M = U + 1e-3 * (rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3)))
    W = O.unitarize(M)
    assert np.abs(W @ W.conj().T - np.eye(3)).max() < 1e-15
    assert abs(np.linalg.det(W) - 1) < 1e-15
    # Gram-Schmidt keeps the direction of row 0
    r0 = M[0] / np.linalg.norm(M[0])
    assert np.abs(W[0] - r0).max() < 1e-15


def test_ta_is_traceless_antihermitian():
    rng = np.random.default_rng(4)
    M = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    A = O.ta(M)
    assert np.abs(A + A.conj().T).max() < 1e-15
    assert abs(np.trace(A)) < 1e-15
    ref = 0.5 * (M - M.conj().T)
    ref -= np.trace(ref) / 3 * np.eye(3)
    assert np.abs(A - ref).max() < 1e-15


# ------------------------------------------------------------------ action
def test_cold_start_plaquette_and_action():
    U = O.gen_cold(DIMS)
    V = np.prod(DIMS)
    p, r = O.plaq_rect(DIMS, U)
    assert p == 18.0 * V and r == 36.0 * V
    assert O.avg_plaquette(DIMS, U) == 1.0
    pr = O.make_params(DIMS, beta=2.25, c1=-0.331)
    _, _, S = O.action(pr, U)
    assert abs(S - 2.25 / 3 * (-(1 + 8 * 0.331) * 18 * V + 0.331 * 36 * V)) < 1e-9
    F = O.force(pr, U)
    assert np.abs(F).max() == 0.0


@pytest.mark.parametrize("n_stout", [0, 2])
def test_gauge_invariance(n_stout):
    U = O.gen_hot(DIMS, 5)
    G = O.gen_hot((*DIMS[:3], DIMS[3]), 6)[:, 0]
    Ug = O.gauge_transform(DIMS, U, np.ascontiguousarray(G))
    p = O.make_params(DIMS, n_stout=n_stout, rho=0.1)
    a, b = O.action(p, U), O.action(p, Ug)
    for x, y in zip(a, b):
        assert abs(x - y) < 1e-11 * max(1.0, abs(x))
    for R, T in ((1, 1), (2, 3)):
        w0, w1 = O.wilson_loop(DIMS, U, (R, 0, 0), T), O.wilson_loop(DIMS, Ug, (R, 0, 0), T)
        assert abs(w0 - w1) < 1e-13


def _fd_check(p, U, site, mu, pair=False, h=1e-5, seed=1):
    dims = tuple(p.dims)
    F = O.force(p, U)
    rng = np.random.default_rng(seed)
    X = rand_herm(rng)

    def S(eps):
        V = U.copy()
        if pair:
            x = np.unravel_index(site, dims[::-1])[::-1]
            y = list(x)
            y[mu] = (y[mu] + 1) % dims[mu]
            s2 = idx(dims, y)
            V[site, mu] = V[site, mu] @ O.expiQ(-X * eps)
            V[s2, mu] = O.expiQ(X * eps) @ V[s2, mu]
        else:
            V[site, mu] = O.expiQ(X * eps) @ V[site, mu]
        return O.action(p, V)[2]

    fd = (S(h) - S(-h)) / (2 * h)
    an = -np.trace(X @ F[site, mu]).real
    return fd, an


@pytest.mark.parametrize("action,n_stout,mag,site,mu,pair", [
    (1, 0, 0, 13, 2, False),   # Iwasaki thin
    (0, 0, 0, 13, 1, False),   # Wilson thin
    (1, 1, 0, 13, 2, False),   # one stout level
    (1, 3, 0, 21, 3, False),   # three stout levels
    (1, 0, 2, 0, 0, True),     # constrained pair (case 10 + case 100)
    (1, 2, 2, 0, 1, True),     # constrained pair through two stout levels
    (0, 1, 2, 1, 2, False),    # free link of a constrained lattice (x0 = 1 is odd)
])
def test_force_is_minus_action_derivative(action, n_stout, mag, site, mu, pair):
    U = O.gen_hot(DIMS, 7)
    p = O.make_params(DIMS, mag=mag, action=action, n_stout=n_stout, rho=0.1)
    fd, an = _fd_check(p, U, site, mu, pair=pair)
    assert abs(fd - an) < 2e-7 * max(1.0, abs(an)), (fd, an)


def test_constrained_last_link_has_no_force():
    U = O.gen_hot(DIMS, 8)
    p = O.make_params(DIMS, mag=2)
    F = O.force(p, U)
    # (x0=1, 0, 0, 0) along mu = 0 is the last link of its segment (case 100)
    assert np.abs(F[idx(DIMS, (1, 0, 0, 0)), 0]).max() == 0.0


# ------------------------------------------------------------------ integrators
def test_force_gradient_is_fourth_order_and_leapfrog_second():
    dims = (4, 4, 4, 4)
    U = O.gen_hot(dims, 9)
    # start from a smoother field so that the MD is in its asymptotic regime
    p0 = O.make_params(dims, mag=0, beta=5.0, n_steps=4)
    P = O.gen_momenta(dims, 1, 0)
    for _ in range(2):
        U, _, _ = O.integrate(p0, U, P * 0.3)
    P = O.gen_momenta(dims, 1, 1)
    res = {}
    for integ in (0, 1):
        dh = []
        for n in (4, 8):
            p = O.make_params(dims, mag=0, beta=5.0, n_steps=n, tau=0.5, integrator=integ)
            h0 = O.hamiltonian(p, U, P)["H"]
            U1, P1, _ = O.integrate(p, U, P)
            dh.append(abs(O.hamiltonian(p, U1, P1)["H"] - h0))
        res[integ] = dh[0] / dh[1]
    assert res[1] > 3.0          # leapfrog: ~ 2^2
    assert res[0] > 10.0         # force gradient: ~ 2^4


@pytest.mark.parametrize("mag,n_stout", [(0, 0), (2, 0), (2, 1)])
def test_reversibility(mag, n_stout):
    dims = (4, 4, 4, 4)
    U = O.gen_hot(dims, 10)
    P = O.gen_momenta(dims, 2, 0)
    p = O.make_params(dims, mag=mag, n_stout=n_stout, n_steps=4, tau=0.5)
    U1, P1, _ = O.integrate(p, U, P)
    U2, P2, _ = O.integrate(p, U1, -P1)
    assert np.abs(U2 - U).max() < 1e-10
    assert np.abs(P2 + P).max() < 1e-9


def test_constrained_plaquette_is_invariant():
    dims = (4, 4, 4, 4)
    U = O.gen_hot(dims, 12)
    P = O.gen_momenta(dims, 3, 0)
    p = O.make_params(dims, mag=2, n_steps=3, tau=0.3)
    c0 = O.constrained_plaquette(dims, U, 2)
    U1, _, _ = O.integrate(p, U, P)
    assert abs(O.constrained_plaquette(dims, U1, 2) - c0) < 1e-12
    assert abs(O.avg_plaquette(dims, U1) - O.avg_plaquette(dims, U)) > 1e-4


def test_wilson_loops_known_values():
    U = O.gen_cold(DIMS)
    assert abs(O.wilson_loop(DIMS, U, (2, 0, 0), 3) - 3.0) < 1e-15
    Uh = O.gen_hot(DIMS, 13)
    # W(1,1) for r = (1,0,0) averages the three (i, t) plaquettes per site
    V = np.prod(DIMS)
    tot = 0.0
    for s in range(V):
        x = np.unravel_index(s, DIMS[::-1])[::-1]
        for i in range(3):
            y = list(x); y[i] = (y[i] + 1) % DIMS[i]
            z = list(x); z[3] = (z[3] + 1) % DIMS[3]
            m = Uh[s, i] @ Uh[idx(DIMS, y), 3] @ Uh[idx(DIMS, z), i].conj().T @ Uh[s, 3].conj().T
            tot += np.trace(m).real
    assert abs(O.wilson_loop(DIMS, Uh, (1, 0, 0), 1) - tot / (3 * V)) < 1e-13


def test_trajectory_metropolis_and_demon_rules():
    dims = (4, 4, 4, 4)
    U = O.gen_hot(dims, 14)
    p = O.make_params(dims, mag=2, n_steps=4)
    P = O.gen_momenta(dims, 4, 0)
    U1, r = O.trajectory(p, 0, U, P, 0.5, [0.0, 0.0])
    assert r["accept"] == (0.5 < np.exp(-r["delta_h"]))
    assert abs(r["delta_h"] - (r["h_new"] - r["h_old"])) < 1e-6
    if not r["accept"]:
        assert np.array_equal(U1, U)
    # demon: window on -sum ReTr changes (field-demon.h:173-186)
    pd = O.make_params(dims, mag=2, n_steps=4, accept=1, e_max=1e9)
    _, rd = O.trajectory(pd, 0, U, P, 0.0, [0.0, 0.0])
    assert rd["accept"] == 1
    assert abs(rd["demon"][0] - (rd["plaq_new"] - rd["plaq_old"])) < 1e-8
    pz = O.make_params(dims, mag=2, n_steps=4, accept=1, e_max=1e-6)
    Uz, rz = O.trajectory(pz, 0, U, P, 0.0, [0.0, 0.0])
    assert rz["accept"] == 0 and rz["demon"] == [0.0, 0.0] and np.array_equal(Uz, U)


def test_demon_sweep_conserves_plaquette_and_rectangle_energy():
    """field-demon.h:25-126: the plaquette and rectangle demons absorb exactly the change
    of the total plaquette / rectangle sums (E_k = -sum dS_k, dS = the action change of
    the loops through the updated link), up to the reunitarisation after each sweep."""
    dims = (4, 4, 4, 4)
    U = O.gen_hot(dims, 3)
    p0, r0 = O.plaq_rect(dims, U)
    U1, E, acc, rej, dev = O.demon_sweeps(dims, U, seed=7, n_sweeps=2, e_max=50.0)
    p1, r1 = O.plaq_rect(dims, U1)
    assert acc + rej == 2 * 2 * 4 * O.volume(dims) and acc > 0 and rej > 0
    assert abs(E[-1, 0] - (p1 - p0)) < 1e-9 and abs(E[-1, 1] - (r1 - r0)) < 1e-9
    assert np.all(np.abs(E) < 50.0) and np.all(dev < 1e-13)
    # the demons never leave the window; with a zero window nothing is accepted
    _, E0, acc0, rej0, _ = O.demon_sweeps(dims, U, seed=7, n_sweeps=1, e_max=0.0)
    assert acc0 == 0 and np.all(E0 == 0.0)


# ------------------------------------------------------------ two-level coupling (field-multi.h)
MDIMS = (4, 4, 4, 8)


def _multi_S(p, rho, eta2, Uf, Uc):
    Zf, Zc = np.zeros_like(Uf), np.zeros_like(Uc)
    return O.multi_hamiltonian(p, rho, eta2, Uf, Zf, Uc, Zc)["H"]


@pytest.mark.parametrize("action", [0, 1])
def test_multi_forces_are_minus_the_coupled_action_derivative(action):
    """get_Fforce / get_Cforce restated (the reference's insertion paths per stout_type, rho and
    eta_sqr as parameters) against a central difference of S_gauge(U) + S_eta(U, C): fine links of
    every stout type (1: all coordinates even, 2: one odd other than mu, 3: mu odd, 4: mu and one
    other odd, 0: not coupled) and coarse links."""
    rng = np.random.default_rng(3)
    Uf, Uc = O.gen_hot(MDIMS, 3), O.gen_hot(O.coarse_dims(MDIMS), 4)
    p = O.make_params(MDIMS, mag=0, action=action, beta=2.25, c1=-0.331)
    rho, eta2 = 0.1, 0.5
    Ff, Fc = O.multi_forces(p, rho, eta2, Uf, Uc)
    h = 1e-5
    # (site, mu): (0,0) type 1, (1,0) type 3, (1,1) type 2, (17,2) type 4, (5,3) type 0, (42,0) type 1
    for field, F, cases in (("fine", Ff, [(0, 0), (1, 0), (1, 1), (17, 2), (5, 3), (42, 0), (85, 3)]),
                            ("coarse", Fc, [(0, 0), (3, 2), (7, 3)])):
        for site, mu in cases:
            X = rand_herm(rng)

            def S(e):
                a, b = Uf.copy(), Uc.copy()
                V = a if field == "fine" else b
                V[site, mu] = O.expiQ(X * e) @ V[site, mu]
                return _multi_S(p, rho, eta2, a, b)

            fd = (S(h) - S(-h)) / (2 * h)
            an = -np.trace(X @ F[site, mu]).real
            assert abs(fd - an) < 2e-7 * max(1.0, abs(an)), (field, site, mu, fd, an)


def test_multi_integrator_is_fourth_order():
    """force_gradient_integrator_multi: |Delta H| falls as dt^4 (16x for half the step)."""
    Uf, Uc = O.gen_hot(MDIMS, 5), O.gen_hot(O.coarse_dims(MDIMS), 6)
    Pf, Pc = O.gen_momenta(MDIMS, 7, 0), O.gen_momenta(O.coarse_dims(MDIMS), 8, 0)
    dh = []
    for n in (4, 8):
        p = O.make_params(MDIMS, mag=0, action=1, beta=2.25, c1=-0.331, tau=0.5, n_steps=n)
        _, _, r = O.multi_trajectory(p, 0.1, 0.5, 0, Uf, Pf, Uc, Pc, 0.0)
        dh.append(abs(r["delta_h"]))
    assert 10.0 < dh[0] / dh[1] < 25.0, dh
