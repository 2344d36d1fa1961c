"""Per-link demon sweep (demon_microcanonical, field-demon.h:25-126): the GPU
sweep against the oracle's sequential restatement on the same links and the
same Philox draws.

Bars: identical accepted / rejected hit counts, demon energies within 1e-9
(sums of O(1) action changes over thousands of hits), swept links within 1e-12,
reunitarisation deviations at rounding level.
"""
import numpy as np
import pytest

import mag_b200 as M
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,e_max", [((4, 4, 4, 4), 50.0), ((4, 4, 4, 6), 20.0), ((2, 4, 2, 4), 8.0)])
def test_demon_sweeps_match_oracle(dims, e_max):
    U = O.gen_hot(dims, 5)
    Uo, Eo, ao, ro, devo = O.demon_sweeps(dims, U, seed=9, n_sweeps=2, e_max=e_max)
    with M.Chmc(dims, mag=0) as c:
        c.set_gauge(U)
        res = c.demon_microcanonical(2, e_max, seed=9, update_links=True)
        Ug = c.get_gauge()
    assert res["accepted"] == ao and res["rejected"] == ro
    assert ao > 0 and ro > 0
    assert np.abs(res["demon_energy"] - Eo).max() < 1e-9
    assert np.all(np.abs(res["demon_energy"]) < e_max)
    assert np.abs(Ug - Uo).max() < 1e-12
    assert np.all(res["reunit_maxdev"] < 1e-13) and np.all(devo < 1e-13)


def test_demon_full_sweep_8x8x8x8():
    """One sweep of all 16384 links of an 8^4 lattice: the site windows are staged over 4096
    site transitions, with periodic wrap-around in every direction."""
    dims = (8, 8, 8, 8)
    U = O.gen_hot(dims, 7)
    Uo, Eo, ao, ro, devo = O.demon_sweeps(dims, U, seed=21, n_sweeps=1, e_max=50.0)
    with M.Chmc(dims, mag=0) as c:
        c.set_gauge(U)
        res = c.demon_microcanonical(1, 50.0, seed=21, update_links=True)
        Ug = c.get_gauge()
    assert res["accepted"] == ao and res["rejected"] == ro
    assert ao + ro == 2 * 4 * 8 ** 4
    assert np.abs(res["demon_energy"] - Eo).max() < 1e-9
    assert np.abs(Ug - Uo).max() < 1e-12


def test_demon_sweep_keeps_links_by_default_and_serves_any_chain():
    chains = [dict(dims=(4, 4, 4, 4)), dict(dims=(4, 4, 6, 4))]
    U1 = O.gen_hot((4, 4, 6, 4), 6)
    Uo, Eo, ao, ro, _ = O.demon_sweeps((4, 4, 6, 4), U1, seed=3, n_sweeps=1, e_max=30.0)
    with M.Chmc(chains=chains, precision="mixed") as c:
        c.hot_start(1)
        U0 = c.get_gauge(0)
        c.set_gauge(U1, chain=1)
        res = c.demon_microcanonical(1, 30.0, seed=3, chain=1)
        assert np.array_equal(c.get_gauge(1), U1) and np.array_equal(c.get_gauge(0), U0)
    assert res["accepted"] == ao and np.abs(res["demon_energy"] - Eo).max() < 1e-9


def test_ensemble_sweeps_each_chain_like_the_oracle():
    """mag_demon_microcanonical_all: every chain of an ensemble swept at once, one CTA per
    chain, chain c drawing with seed + its stream index."""
    dims = [(4, 4, 4, 4), (4, 4, 4, 6), (2, 4, 2, 4)]
    hot = [O.gen_hot(d, 11 + c) for c, d in enumerate(dims)]
    with M.Chmc(chains=[dict(dims=d, mag=0) for d in dims]) as c:
        c.set_stream_index([5, 6, 7])
        for k, U in enumerate(hot):
            c.set_gauge(U, chain=k)
        res = c.demon_microcanonical_all(2, 30.0, seed=9, update_links=True)
        Ug = [c.get_gauge(k) for k in range(len(dims))]
    for k, d in enumerate(dims):
        Uo, Eo, ao, ro, devo = O.demon_sweeps(d, hot[k], seed=9 + 5 + k, n_sweeps=2, e_max=30.0)
        assert res[k]["accepted"] == ao and res[k]["rejected"] == ro
        assert np.abs(res[k]["demon_energy"] - Eo).max() < 1e-9
        assert np.abs(Ug[k] - Uo).max() < 1e-12
        assert np.all(res[k]["reunit_maxdev"] < 1e-13)


def test_ensemble_sweeps_keep_links_by_default():
    dims = [(4, 4, 4, 4), (2, 4, 2, 4)]
    with M.Chmc(chains=[dict(dims=d, mag=0) for d in dims]) as c:
        c.hot_start(3)
        U0 = [c.get_gauge(k) for k in range(2)]
        res = c.demon_microcanonical_all(1, 30.0, seed=2)
        assert all(np.array_equal(c.get_gauge(k), U0[k]) for k in range(2))
    assert all(r["accepted"] + r["rejected"] == 2 * 4 * int(np.prod(d)) for r, d in zip(res, dims))


def test_zero_window_accepts_nothing():
    U = O.gen_hot((4, 4, 4, 4), 2)
    with M.Chmc((4, 4, 4, 4), mag=0) as c:
        c.set_gauge(U)
        res = c.demon_microcanonical(1, 0.0, seed=1)
    assert res["accepted"] == 0 and res["rejected"] == 2 * 4 * 256
    assert np.all(res["demon_energy"] == 0.0)
