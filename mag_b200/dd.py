"""One lattice split into slabs along x3 (domain decomposition with halo exchange).

``DomainChmc`` mirrors the part of ``Chmc`` that run_chmc needs (field-hmc.h:770-857)
for a lattice held as ``nshards`` slabs of dims[3] / nshards time slices, each an
ordinary context over its slices plus ``halo`` slices of its neighbours.  The
reference keeps such a slab per MPI rank in a qlat Field with an expanded Geometry
(expansion(2, 2, 2, 2), field-hmc.h:777-781) and refreshes its halo with
fetch_expanded_chart before every force (field-hmc.h:544-558); here the halos are
refreshed after every kernel whose output is read across a slab boundary (links,
each stout level, the double links, each level's Lambda), the sums of
get_hamiltonian are added over the slabs (its MPI_Allreduce, field-hmc.h:628) and
every slab takes the same accept decision (the MPI_Bcast of field-hmc.h:823).

Fields cross this interface in the lattice's host layout (V, 4, 3, 3) complex128,
the layout ``Chmc`` uses for an undivided lattice.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import MagParams, TrajResult, check
from .field_hmc import _dp, make_params, volume


class DomainChmc:
    def __init__(self, dims, nshards: int, halo: int = 2, **kw):
        self._lib = _lib.load()
        self.dims = tuple(int(d) for d in dims)
        self.nshards, self.halo = int(nshards), int(halo)
        p = make_params(self.dims, **kw)
        h = ctypes.c_void_p()
        check(self._lib.mag_dd_create(ctypes.byref(p), self.nshards, self.halo, ctypes.byref(h)), "mag_dd_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.mag_dd_destroy(self._h)
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

    def _field(self) -> np.ndarray:
        return np.zeros((volume(self.dims), 4, 3, 3), np.complex128)

    def _in(self, F: np.ndarray) -> np.ndarray:
        F = np.ascontiguousarray(F, np.complex128)
        assert F.shape == (volume(self.dims), 4, 3, 3)
        return F

    def set_gauge(self, U: np.ndarray) -> None:
        check(self._lib.mag_dd_gauge_set(self._h, _dp(self._in(U))), "mag_dd_gauge_set")

    def get_gauge(self) -> np.ndarray:
        U = self._field()
        check(self._lib.mag_dd_gauge_get(self._h, _dp(U)), "mag_dd_gauge_get")
        return U

    def init_momentum(self, P: np.ndarray) -> None:
        check(self._lib.mag_dd_momentum_set(self._h, _dp(self._in(P))), "mag_dd_momentum_set")

    def get_momentum(self) -> np.ndarray:
        P = self._field()
        check(self._lib.mag_dd_momentum_get(self._h, _dp(P)), "mag_dd_momentum_get")
        return P

    def hot_start(self, seed: int) -> None:
        check(self._lib.mag_dd_hot_start(self._h, int(seed)), "mag_dd_hot_start")

    def set_uniforms(self, u) -> None:
        if u is None:
            check(self._lib.mag_dd_uniforms_set(self._h, None), "mag_dd_uniforms_set")
            return
        a = np.ascontiguousarray(np.asarray(u, np.float64).reshape(1))
        check(self._lib.mag_dd_uniforms_set(self._h, _dp(a)), "mag_dd_uniforms_set")

    def get_force(self) -> np.ndarray:
        F = self._field()
        check(self._lib.mag_dd_gauge_force(self._h, _dp(F)), "mag_dd_gauge_force")
        return F

    def trajectory(self, refresh_momenta: bool = True) -> dict:
        r = TrajResult()
        check(self._lib.mag_dd_trajectory(self._h, 1 if refresh_momenta else 0, ctypes.byref(r)),
              "mag_dd_trajectory")
        return r.as_dict()


__all__ = ["DomainChmc", "MagParams"]
