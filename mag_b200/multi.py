"""Two-level coupling of field-multi.h: a fine lattice and a coarse lattice of half its extent.

``MultiChmc`` mirrors run_hmc_multi (field-multi.h:758-900): the coarse field C is
coupled to the stout-smeared blocked links of the fine field U through
    S_eta = -1/eta_sqr sum_{coarse x, mu} ReTr(C(x,mu)^dag e^{iQ(2x,mu)} V(2x,mu)),
V(y,mu) = U(y,mu) U(y+mu,mu), Q = -i rho TA(stp V^dag) with stp the staple of the 2-link
(get_U, get_Q, get_staple_rect); H = K_fine + K_coarse + S_gauge(U) + S_eta and one
force-gradient trajectory moves both fields (force_gradient_integrator_multi).  The
reference reads rho and eta_sqr from globals outside its tree; here they are parameters.
Fields are (V, 4, 3, 3) complex128 arrays, as for ``Chmc``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check
from .field_hmc import _dp, make_params, volume


class MultiChmc:
    def __init__(self, dims, rho: float = 0.1, eta_sqr: float = 1.0, **kw):
        self._lib = _lib.load()
        self.dims = tuple(int(d) for d in dims)
        self.coarse_dims = tuple(d // 2 for d in self.dims)
        self.rho, self.eta_sqr = float(rho), float(eta_sqr)
        p = make_params(self.dims, **{**kw, "mag": 0})
        h = ctypes.c_void_p()
        check(self._lib.mag_multi_create(ctypes.byref(p), self.rho, self.eta_sqr, ctypes.byref(h)),
              "mag_multi_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.mag_multi_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _pair(self):
        return (np.zeros((volume(self.dims), 4, 3, 3), np.complex128),
                np.zeros((volume(self.coarse_dims), 4, 3, 3), np.complex128))

    @staticmethod
    def _c(a):
        return np.ascontiguousarray(a, np.complex128)

    def set_gauge(self, Uf, Uc) -> None:
        check(self._lib.mag_multi_gauge_set(self._h, _dp(self._c(Uf)), _dp(self._c(Uc))), "mag_multi_gauge_set")

    def get_gauge(self):
        f, c = self._pair()
        check(self._lib.mag_multi_gauge_get(self._h, _dp(f), _dp(c)), "mag_multi_gauge_get")
        return f, c

    def init_momentum(self, Pf, Pc) -> None:
        check(self._lib.mag_multi_momentum_set(self._h, _dp(self._c(Pf)), _dp(self._c(Pc))),
              "mag_multi_momentum_set")

    def get_forces(self):
        """(fine force, coarse force): get_Fforce and get_Cforce of the current fields."""
        f, c = self._pair()
        check(self._lib.mag_multi_forces(self._h, _dp(f), _dp(c)), "mag_multi_forces")
        return f, c

    def get_hamiltonian(self) -> dict:
        out = (ctypes.c_double * 4)()
        check(self._lib.mag_multi_hamiltonian(self._h, out), "mag_multi_hamiltonian")
        return {"H": out[0], "kinetic": out[1], "fine": out[2], "eta": out[3]}

    def trajectory(self, uniform: float, traj_index: int = 0) -> dict:
        out = (ctypes.c_double * 6)()
        check(self._lib.mag_multi_trajectory(self._h, int(traj_index), float(uniform), out), "mag_multi_trajectory")
        return {"h_old": out[0], "h_new": out[1], "delta_h": out[2], "accept": int(out[3]),
                "reunit_fine": out[4], "reunit_coarse": out[5]}


__all__ = ["MultiChmc"]
