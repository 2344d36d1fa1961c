"""Two-level coupling (field-multi.h) on the GPU against the oracle.

mag_multi_* (kernels_multi.cu): the coarse-link kernel forms the blocked link V,
its 2-link staple, Q and e^{iQ}, the coupling energy, the coarse force and Lambda;
the fine-link kernel adds the coupling's derivative (the reference's insertion
paths per stout_type) to the fine gauge force.  Against the oracle's literal
restatement (itself checked against a finite difference of the coupled action in
tests/test_oracle.py): forces to 1e-11 relative, Hamiltonian parts to 1e-12
relative, and trajectories (both fields moved by the force-gradient integrator)
to Delta H 1e-9 with the same accept bit and fields to 1e-10.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

MDIMS = (4, 4, 4, 8)


def maxrel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


@pytest.mark.parametrize("action", ["wilson", "iwasaki"])
def test_multi_forces_and_hamiltonian_match_the_oracle(action):
    from mag_b200.multi import MultiChmc

    cd = O.coarse_dims(MDIMS)
    Uf, Uc = O.gen_hot(MDIMS, 3), O.gen_hot(cd, 4)
    Pf, Pc = O.gen_momenta(MDIMS, 5, 0), O.gen_momenta(cd, 6, 0)
    a = 1 if action == "iwasaki" else 0
    p = O.make_params(MDIMS, mag=0, action=a, beta=2.25, c1=-0.331)
    Ff_o, Fc_o = O.multi_forces(p, 0.1, 0.5, Uf, Uc)
    ho = O.multi_hamiltonian(p, 0.1, 0.5, Uf, Pf, Uc, Pc)
    with MultiChmc(MDIMS, rho=0.1, eta_sqr=0.5, action=action, beta=2.25, c1=-0.331) as m:
        m.set_gauge(Uf, Uc)
        m.init_momentum(Pf, Pc)
        Ff, Fc = m.get_forces()
        h = m.get_hamiltonian()
    assert maxrel(Ff, Ff_o) < 1e-11
    assert maxrel(Fc, Fc_o) < 1e-11
    for k in ("H", "kinetic", "fine", "eta"):
        assert abs(h[k] - ho[k]) <= 1e-12 * max(1.0, abs(ho[k])), (k, h[k], ho[k])


@pytest.mark.parametrize("action,n_steps", [("iwasaki", 4), ("wilson", 6)])
def test_multi_trajectories_match_the_oracle(action, n_steps):
    from mag_b200.multi import MultiChmc

    cd = O.coarse_dims(MDIMS)
    Uf, Uc = O.gen_hot(MDIMS, 7), O.gen_hot(cd, 8)
    a = 1 if action == "iwasaki" else 0
    p = O.make_params(MDIMS, mag=0, action=a, beta=2.25, c1=-0.331, tau=1.0, n_steps=n_steps)
    with MultiChmc(MDIMS, rho=0.1, eta_sqr=0.5, action=action, beta=2.25, c1=-0.331, tau=1.0,
                   n_steps=n_steps) as m:
        m.set_gauge(Uf, Uc)
        Uof, Uoc = Uf, Uc
        for t in range(2):
            Pf, Pc = O.gen_momenta(MDIMS, 9, t), O.gen_momenta(cd, 10, t)
            u = O.gen_uniform(9, t)
            m.init_momentum(Pf, Pc)
            g = m.trajectory(u, t)
            Uof, Uoc, o = O.multi_trajectory(p, 0.1, 0.5, t, Uof, Pf, Uoc, Pc, u)
            assert g["accept"] == o["accept"]
            assert abs(g["h_old"] - o["h_old"]) <= 1e-12 * abs(o["h_old"])
            assert abs(g["delta_h"] - o["delta_h"]) < 1e-9, (g["delta_h"], o["delta_h"])
            gf, gc = m.get_gauge()
            assert np.abs(gf - Uof).max() < 1e-10 and np.abs(gc - Uoc).max() < 1e-10
