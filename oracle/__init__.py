"""ctypes front end of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this package, and only as the checker.  The product library never calls
it.  Parity is unpinned against reference outputs (the reference has no golden
vectors and cannot be built here); the oracle is pinned by invariants instead.

Fields are numpy arrays of shape (V, 4, 3, 3) complex128 (host AoS, x fastest),
i.e. the memory layout ``double[V][4][3][3][2]`` of the reference's
``Field<cps::Matrix>`` with multiplicity 4.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libmag_oracle.so")
_lib = None


class Params(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int * 4),
        ("mag", ctypes.c_int),
        ("action", ctypes.c_int),
        ("beta", ctypes.c_double),
        ("c1", ctypes.c_double),
        ("rho", ctypes.c_double),
        ("n_stout", ctypes.c_int),
        ("tau", ctypes.c_double),
        ("n_steps", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("accept", ctypes.c_int),
        ("e_max", ctypes.c_double),
        ("n_forced", ctypes.c_int),
    ]


class Traj(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "h_old", "h_new", "delta_h", "kin_old", "kin_new", "pot_old", "pot_new",
        "plaq_old", "plaq_new", "rect_old", "rect_new", "uniform")] + [
        ("demon", ctypes.c_double * 2),
        ("reunit_maxdev", ctypes.c_double),
        ("avg_plaquette", ctypes.c_double),
        ("accept", ctypes.c_int),
    ]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["demon"] = [self.demon[0], self.demon[1]]
        return d


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (system g++ + OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "mag_oracle.cpp"))):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        pp = ctypes.POINTER(Params)
        sig = {
            "mo_set_threads": (None, [ctypes.c_int]),
            "mo_get_threads": (ctypes.c_int, []),
            "mo_philox4x32": (None, [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                     ctypes.POINTER(ctypes.c_uint32)]),
            "mo_gen_hot": (None, [ip, ctypes.c_uint64, dp]),
            "mo_gen_momenta": (None, [ip, ctypes.c_uint64, ctypes.c_uint64, dp]),
            "mo_gen_uniform": (ctypes.c_double, [ctypes.c_uint64, ctypes.c_uint64]),
            "mo_expiQ": (None, [dp, dp]),
            "mo_dexpiQ": (None, [dp, dp, dp]),
            "mo_compute_lambda": (None, [dp, dp, dp, dp]),
            "mo_unitarize": (None, [dp]),
            "mo_ta": (None, [dp, dp]),
            "mo_plaq_rect": (None, [ip, dp, dp]),
            "mo_avg_plaquette": (ctypes.c_double, [ip, dp]),
            "mo_action": (None, [pp, dp, dp]),
            "mo_kinetic": (ctypes.c_double, [pp, dp]),
            "mo_staple_dagger": (None, [pp, dp, dp]),
            "mo_force": (None, [pp, dp, dp]),
            "mo_evolve_gauge": (None, [pp, dp, dp, ctypes.c_double]),
            "mo_evolve_momentum": (None, [ip, dp, dp, ctypes.c_double, ctypes.c_double]),
            "mo_reunitarize": (ctypes.c_double, [ip, dp]),
            "mo_integrate": (None, [pp, dp, dp, dp]),
            "mo_hamiltonian": (None, [pp, dp, dp, dp]),
            "mo_trajectory": (None, [pp, ctypes.c_int, dp, dp, ctypes.c_double, dp, ctypes.POINTER(Traj)]),
            "mo_run": (None, [pp, ctypes.c_uint64, ctypes.c_int, dp, ctypes.POINTER(Traj)]),
            "mo_stout_forward": (None, [pp, dp, dp]),
            "mo_wilson_loop": (ctypes.c_double, [ip, dp, ip, ctypes.c_int]),
            "mo_constrained_plaquette": (ctypes.c_double, [ip, dp, ctypes.c_int]),
            "mo_gauge_transform": (None, [ip, dp, dp]),
            "mo_demon_sweeps": (None, [ip, dp, ctypes.c_uint64, ctypes.c_int, ctypes.c_double, dp,
                                       ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), dp]),
            "mo_multi_forces": (None, [pp, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp]),
            "mo_multi_hamiltonian": (None, [pp, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp, dp]),
            "mo_multi_trajectory": (None, [pp, ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp, dp, dp,
                                           ctypes.c_double, dp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


# ------------------------------------------------------------------ helpers
def _dp(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _dims(dims):
    return (ctypes.c_int * 4)(*[int(d) for d in dims])


def volume(dims) -> int:
    v = 1
    for d in dims:
        v *= int(d)
    return v


def new_field(dims) -> np.ndarray:
    return np.zeros((volume(dims), 4, 3, 3), dtype=np.complex128)


def make_params(dims, mag=2, action=1, beta=2.25, c1=-0.331, rho=0.1, n_stout=0, tau=1.0, n_steps=8,
                integrator=0, accept=0, e_max=100.0, n_forced=0) -> Params:
    p = Params()
    p.dims[:] = [int(d) for d in dims]
    p.mag, p.action, p.beta, p.c1, p.rho, p.n_stout = mag, action, beta, c1, rho, n_stout
    p.tau, p.n_steps, p.integrator, p.accept, p.e_max, p.n_forced = tau, n_steps, integrator, accept, e_max, n_forced
    return p


def set_threads(n: int) -> None:
    lib().mo_set_threads(int(n))


def philox4x32(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().mo_philox4x32(c, k, o)
    return [int(v) for v in o]


def gen_hot(dims, seed: int) -> np.ndarray:
    U = new_field(dims)
    lib().mo_gen_hot(_dims(dims), seed, _dp(U))
    return U


def gen_cold(dims) -> np.ndarray:
    U = new_field(dims)
    U[:, :] = np.eye(3)
    return U


def gen_momenta(dims, seed: int, traj: int) -> np.ndarray:
    P = new_field(dims)
    lib().mo_gen_momenta(_dims(dims), seed, traj, _dp(P))
    return P


def gen_uniform(seed: int, traj: int) -> float:
    return lib().mo_gen_uniform(seed, traj)


def _m(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def expiQ(Q):
    out = np.zeros((3, 3), np.complex128)
    lib().mo_expiQ(_dp(_m(Q)), _dp(out))
    return out


def dexpiQ(Q, DQ):
    out = np.zeros((3, 3), np.complex128)
    lib().mo_dexpiQ(_dp(_m(Q)), _dp(_m(DQ)), _dp(out))
    return out


def compute_lambda(Q, S, U):
    out = np.zeros((3, 3), np.complex128)
    lib().mo_compute_lambda(_dp(_m(Q)), _dp(_m(S)), _dp(_m(U)), _dp(out))
    return out


def unitarize(M):
    m = _m(M).copy()
    lib().mo_unitarize(_dp(m))
    return m


def ta(M):
    out = np.zeros((3, 3), np.complex128)
    lib().mo_ta(_dp(_m(M)), _dp(out))
    return out


def plaq_rect(dims, U):
    out = (ctypes.c_double * 2)()
    lib().mo_plaq_rect(_dims(dims), _dp(U), out)
    return out[0], out[1]


def avg_plaquette(dims, U):
    return lib().mo_avg_plaquette(_dims(dims), _dp(U))


def action(p: Params, U):
    out = (ctypes.c_double * 3)()
    lib().mo_action(ctypes.byref(p), _dp(U), out)
    return out[0], out[1], out[2]


def kinetic(p: Params, P):
    return lib().mo_kinetic(ctypes.byref(p), _dp(P))


def staple_dagger(p: Params, U):
    V = np.zeros_like(U)
    lib().mo_staple_dagger(ctypes.byref(p), _dp(U), _dp(V))
    return V


def force(p: Params, U):
    F = np.zeros_like(U)
    lib().mo_force(ctypes.byref(p), _dp(U), _dp(F))
    return F


def evolve_gauge(p: Params, U, P, dt):
    U = U.copy()
    lib().mo_evolve_gauge(ctypes.byref(p), _dp(U), _dp(P), dt)
    return U


def evolve_momentum(dims, P, F, dt, m=1.0):
    P = P.copy()
    lib().mo_evolve_momentum(_dims(dims), _dp(P), _dp(F), dt, m)
    return P


def reunitarize(dims, U):
    U = U.copy()
    d = lib().mo_reunitarize(_dims(dims), _dp(U))
    return U, d


def integrate(p: Params, U, P):
    U = U.copy()
    P = P.copy()
    d = ctypes.c_double()
    lib().mo_integrate(ctypes.byref(p), _dp(U), _dp(P), ctypes.byref(d))
    return U, P, d.value


def hamiltonian(p: Params, U, P):
    out = (ctypes.c_double * 5)()
    lib().mo_hamiltonian(ctypes.byref(p), _dp(U), _dp(P), out)
    return {"H": out[0], "kinetic": out[1], "action": out[2], "plaq": out[3], "rect": out[4]}


def trajectory(p: Params, traj_index, U, P, uniform, demon):
    U = U.copy()
    d = (ctypes.c_double * 2)(*demon)
    r = Traj()
    lib().mo_trajectory(ctypes.byref(p), traj_index, _dp(U), _dp(P), uniform, d, ctypes.byref(r))
    return U, r.as_dict()


def run(p: Params, seed: int, n_traj: int, U):
    U = U.copy()
    res = (Traj * n_traj)()
    lib().mo_run(ctypes.byref(p), seed, n_traj, _dp(U), res)
    return U, [r.as_dict() for r in res]


def stout_forward(p: Params, U):
    out = np.zeros((p.n_stout + 1,) + U.shape, np.complex128)
    lib().mo_stout_forward(ctypes.byref(p), _dp(U), _dp(out))
    return out


def wilson_loop(dims, U, r, T):
    rr = (ctypes.c_int * 3)(*[int(v) for v in r])
    return lib().mo_wilson_loop(_dims(dims), _dp(U), rr, int(T))


def constrained_plaquette(dims, U, mag):
    return lib().mo_constrained_plaquette(_dims(dims), _dp(U), int(mag))


def gauge_transform(dims, U, G):
    U = U.copy()
    lib().mo_gauge_transform(_dims(dims), _dp(U), _dp(_m(G)))
    return U


def demon_sweeps(dims, U, seed: int, n_sweeps: int, e_max: float):
    """field-demon.h:25-126 demon_microcanonical: returns (U after the sweeps, demon
    energies [n_sweeps, 4], accepted hits, rejected hits, reunitarize deviation per sweep)."""
    U = np.ascontiguousarray(U, np.complex128).copy()
    E = np.zeros((n_sweeps, 4))
    dev = np.zeros(n_sweeps)
    a, r = ctypes.c_int64(), ctypes.c_int64()
    lib().mo_demon_sweeps(_dims(dims), _dp(U), int(seed), int(n_sweeps), float(e_max), _dp(E), ctypes.byref(a),
                          ctypes.byref(r), _dp(dev))
    return U, E, a.value, r.value, dev


# ------------------------------------------------------------ two-level coupling
def coarse_dims(dims):
    return tuple(int(d) // 2 for d in dims)


def multi_forces(p: Params, rho: float, eta_sqr: float, Uf, Uc):
    """field-multi.h get_Fforce / get_Cforce: (fine force, coarse force)."""
    Ff, Fc = np.zeros_like(Uf), np.zeros_like(Uc)
    lib().mo_multi_forces(ctypes.byref(p), rho, eta_sqr, _dp(_m4(Uf)), _dp(_m4(Uc)), _dp(Ff), _dp(Fc))
    return Ff, Fc


def multi_hamiltonian(p: Params, rho: float, eta_sqr: float, Uf, Pf, Uc, Pc):
    """field-multi.h get_hamiltonian_multi: {H, kinetic, fine action, coupling}."""
    out = (ctypes.c_double * 4)()
    lib().mo_multi_hamiltonian(ctypes.byref(p), rho, eta_sqr, _dp(_m4(Uf)), _dp(_m4(Pf)), _dp(_m4(Uc)),
                               _dp(_m4(Pc)), out)
    return {"H": out[0], "kinetic": out[1], "fine": out[2], "eta": out[3]}


def multi_trajectory(p: Params, rho: float, eta_sqr: float, traj_index: int, Uf, Pf, Uc, Pc, uniform: float):
    """One run_hmc_multi trajectory with given momenta and uniform: (Uf, Uc, record)."""
    Uf, Uc = _m4(Uf).copy(), _m4(Uc).copy()
    out = (ctypes.c_double * 6)()
    lib().mo_multi_trajectory(ctypes.byref(p), rho, eta_sqr, int(traj_index), _dp(Uf), _dp(_m4(Pf)), _dp(Uc),
                              _dp(_m4(Pc)), uniform, out)
    return Uf, Uc, {"h_old": out[0], "h_new": out[1], "delta_h": out[2], "accept": int(out[3]),
                    "reunit_fine": out[4], "reunit_coarse": out[5]}


def _m4(a):
    return np.ascontiguousarray(a, dtype=np.complex128)

