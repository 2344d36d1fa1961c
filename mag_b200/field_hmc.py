"""Host-side mirror of mag's field-*.h operator surface over libmag_b200.so.

The reference is header-only C++ (field-hmc.h, field-matrix.h, field-multi.h,
field-wloop.h, field-demon.h) with free functions over ``Field<cps::Matrix>``.
Here one ``Chmc`` object owns the device fields of one lattice (or of an
ensemble of chains) and exposes the same operations under the same names;
fields cross the boundary as numpy arrays of shape (V, 4, 3, 3) complex128,
the reference's AoS layout with x0 fastest.

Errors raise ``MagError`` (the reference asserts and aborts).
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import MagParams, TrajResult, check

_ACTIONS = {"wilson": _lib.ACTION_WILSON, "iwasaki": _lib.ACTION_IWASAKI}
_PREC = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}
_INTEG = {"fg": _lib.INT_FORCE_GRADIENT, "force_gradient": _lib.INT_FORCE_GRADIENT,
          "leapfrog": _lib.INT_LEAPFROG}
_ACCEPT = {"metropolis": _lib.ACCEPT_METROPOLIS, "demon": _lib.ACCEPT_DEMON}


def volume(dims: Sequence[int]) -> int:
    v = 1
    for d in dims:
        v *= int(d)
    return v


def make_params(dims, mag=2, action="iwasaki", beta=2.25, c1=-0.331, rho=0.1, n_stout=0, tau=1.0, n_steps=8,
                precision="fp64", integrator="fg", accept="metropolis", e_max=100.0, n_forced_accept=0,
                seed=1) -> MagParams:
    """Arg_chmc (field-hmc.h:294-307) + qlat::Gauge + run options."""
    p = MagParams()
    p.dims[:] = [int(d) for d in dims]
    p.mag = int(mag)
    p.action = _ACTIONS[action] if isinstance(action, str) else int(action)
    p.beta, p.c1, p.rho = float(beta), float(c1), float(rho)
    p.n_stout = int(n_stout)
    p.tau, p.n_steps = float(tau), int(n_steps)
    p.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
    p.integrator = _INTEG[integrator] if isinstance(integrator, str) else int(integrator)
    p.accept = _ACCEPT[accept] if isinstance(accept, str) else int(accept)
    p.e_max = float(e_max)
    p.n_forced_accept = int(n_forced_accept)
    p.seed = int(seed)
    return p


def _dp(a: np.ndarray):
    assert a.dtype == np.complex128 or a.dtype == np.float64
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Chmc:
    """Device-resident constrained HMC state (run_chmc's fields, field-hmc.h:770-784)."""

    def __init__(self, dims=None, *, chains: Iterable[dict] | None = None, **kw):
        self._lib = _lib.load()
        if chains is None:
            plist = [make_params(dims, **kw)]
        else:
            plist = [make_params(**{**kw, **c}) for c in chains]
        self.params = plist
        self.dims = [tuple(p.dims) for p in plist]
        arr = (MagParams * len(plist))(*plist)
        h = ctypes.c_void_p()
        check(self._lib.mag_ensemble_create(arr, len(plist), ctypes.byref(h)), "mag_ensemble_create")
        self._h = h
        self.n_chains = len(plist)

    # ------------------------------------------------------------ lifecycle
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.mag_ctx_destroy(self._h)
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

    def volume(self, chain: int = 0) -> int:
        return volume(self.dims[chain])

    def _field(self, chain: int) -> np.ndarray:
        return np.zeros((self.volume(chain), 4, 3, 3), np.complex128)

    def _out_field(self, chain: int, out: np.ndarray | None) -> np.ndarray:
        if out is None:
            return self._field(chain)
        shape = (self.volume(chain), 4, 3, 3)
        if out.shape != shape or out.dtype != np.complex128 or not out.flags.c_contiguous or not out.flags.writeable:
            raise ValueError(f"out must be a writeable C-contiguous complex128 array of shape {shape}")
        return out

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        check(self._lib.mag_ctx_device_bytes(self._h, ctypes.byref(b)), "mag_ctx_device_bytes")
        return b.value

    # ------------------------------------------------------------ field I/O
    def set_gauge(self, U: np.ndarray, chain: int = 0) -> None:
        U = np.ascontiguousarray(U, np.complex128)
        assert U.shape == (self.volume(chain), 4, 3, 3)
        check(self._lib.mag_gauge_set(self._h, chain, _dp(U)), "mag_gauge_set")

    def get_gauge(self, chain: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """The links of ``chain``; ``out`` (C-contiguous complex128, shape (V,4,3,3)),
        e.g. a pinned buffer, receives them in place of a new array."""
        U = self._out_field(chain, out)
        check(self._lib.mag_gauge_get(self._h, chain, _dp(U)), "mag_gauge_get")
        return U

    def set_stream_index(self, index: Sequence[int]) -> None:
        """Philox stream of each chain (key = seed + index[c]); see mag_set_stream_index."""
        a = (ctypes.c_int64 * self.n_chains)(*[int(i) for i in index])
        check(self._lib.mag_set_stream_index(self._h, a), "mag_set_stream_index")

    def hot_start(self, seed: int) -> None:
        check(self._lib.mag_gauge_hot_start(self._h, int(seed)), "mag_gauge_hot_start")

    def cold_start(self) -> None:
        check(self._lib.mag_gauge_cold_start(self._h), "mag_gauge_cold_start")

    def init_momentum(self, P: np.ndarray | None = None, chain: int = 0, traj: int = 0) -> None:
        """init_momentum (field-hmc.h:675): host momenta, or Philox momenta of trajectory ``traj``."""
        if P is None:
            check(self._lib.mag_momentum_refresh(self._h, int(traj)), "mag_momentum_refresh")
            return
        P = np.ascontiguousarray(P, np.complex128)
        check(self._lib.mag_momentum_set(self._h, chain, _dp(P)), "mag_momentum_set")

    def get_momentum(self, chain: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        P = self._out_field(chain, out)
        check(self._lib.mag_momentum_get(self._h, chain, _dp(P)), "mag_momentum_get")
        return P

    def set_uniforms(self, u: Sequence[float] | None) -> None:
        if u is None:
            check(self._lib.mag_uniforms_set(self._h, None), "mag_uniforms_set")
            return
        a = np.ascontiguousarray(np.asarray(u, np.float64).reshape(self.n_chains))
        check(self._lib.mag_uniforms_set(self._h, _dp(a)), "mag_uniforms_set")

    # ------------------------------------------------------------ operators
    def get_force(self, chain: int = 0) -> np.ndarray:
        """get_force (field-hmc.h:339-425), through the stout chain when n_stout > 0."""
        F = self._field(chain)
        check(self._lib.mag_gauge_force(self._h, chain, _dp(F)), "mag_gauge_force")
        return F

    def get_extended_staple_dagger(self, chain: int = 0) -> np.ndarray:
        """get_extended_staple_dagger (field-hmc.h:262-269) of every link of the smeared field."""
        V = self._field(chain)
        check(self._lib.mag_staple(self._h, chain, _dp(V)), "mag_staple")
        return V

    def gauge_action(self, chain: int = 0):
        """(total_plaq, total_rectangular, S) of the smeared links (field-matrix.h:299-385, field-hmc.h:632-639)."""
        p, r, s = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(self._lib.mag_action(self._h, chain, ctypes.byref(p), ctypes.byref(r), ctypes.byref(s)), "mag_action")
        return p.value, r.value, s.value

    def total_plaq(self, chain: int = 0) -> float:
        return self.gauge_action(chain)[0]

    def total_rectangular(self, chain: int = 0) -> float:
        return self.gauge_action(chain)[1]

    def avg_plaquette(self, chain: int = 0) -> float:
        v = ctypes.c_double()
        check(self._lib.mag_plaquette(self._h, chain, ctypes.byref(v)), "mag_plaquette")
        return v.value

    def kinetic_energy(self, chain: int = 0) -> float:
        v = ctypes.c_double()
        check(self._lib.mag_kinetic(self._h, chain, ctypes.byref(v)), "mag_kinetic")
        return v.value

    def get_hamiltonian(self, chain: int = 0):
        """get_hamiltonian (field-hmc.h:589-644): returns (H, [kinetic, potential])."""
        out = np.zeros(3)
        check(self._lib.mag_hamiltonian(self._h, chain, _dp(out)), "mag_hamiltonian")
        return float(out[0]), [float(out[1]), float(out[2])]

    def evolve_gauge_field(self, dt: float, src: str = "momenta") -> None:
        """evolve_gauge_field (field-hmc.h:442-482) with the momenta, or with the force of the
        current links (src="force": the force-gradient step's U <- exp(i dt F(U)) U)."""
        if src == "momenta":
            check(self._lib.mag_evolve_gauge(self._h, float(dt)), "mag_evolve_gauge")
        else:
            code = {"force": 1}[src]
            check(self._lib.mag_evolve_gauge_src(self._h, float(dt), code), "mag_evolve_gauge_src")

    def evolve_momentum(self, dt: float) -> None:
        check(self._lib.mag_evolve_momentum(self._h, float(dt)), "mag_evolve_momentum")

    def force_gradient_integrator(self) -> None:
        """force_gradient_integrator (field-hmc.h:525-567) or leap_frog_integrator per the params."""
        check(self._lib.mag_integrate(self._h), "mag_integrate")

    def reunitarize(self) -> list:
        out = np.zeros(self.n_chains)
        check(self._lib.mag_reunitarize(self._h, _dp(out)), "mag_reunitarize")
        return [float(v) for v in out]

    def stout_level(self, level: int, chain: int = 0) -> np.ndarray:
        U = self._field(chain)
        check(self._lib.mag_stout_level(self._h, chain, int(level), _dp(U)), "mag_stout_level")
        return U

    # ------------------------------------------------------------ HMC
    def trajectory(self, refresh_momenta: bool = True) -> list:
        """One run_chmc trajectory (field-hmc.h:806-843) of every chain."""
        res = (TrajResult * self.n_chains)()
        check(self._lib.mag_trajectory(self._h, 1 if refresh_momenta else 0, res), "mag_trajectory")
        return [r.as_dict() for r in res]

    def run_chmc(self, n_traj: int) -> list:
        """n trajectories replayed as CUDA graphs; returns [traj][chain] records."""
        res = (TrajResult * (n_traj * self.n_chains))()
        check(self._lib.mag_run(self._h, int(n_traj), res), "mag_run")
        return [[res[t * self.n_chains + c].as_dict() for c in range(self.n_chains)] for t in range(n_traj)]

    def traj_counter(self) -> int:
        v = ctypes.c_int64()
        check(self._lib.mag_traj_counter(self._h, ctypes.byref(v)), "mag_traj_counter")
        return v.value

    def set_traj_counter(self, t: int) -> None:
        check(self._lib.mag_set_traj_counter(self._h, int(t)), "mag_set_traj_counter")

    # ------------------------------------------------------------ measurement
    def avg_wilson_loop(self, r: Sequence[int], T: int, chain: int = 0) -> float:
        """avg_wilson_loop (field-wloop.h:58-99)."""
        rr = (ctypes.c_int * 3)(*[int(v) for v in r])
        v = ctypes.c_double()
        check(self._lib.mag_wilson_loop(self._h, chain, rr, int(T), ctypes.byref(v)), "mag_wilson_loop")
        return v.value

    def wilson_loops(self, Rmax: int, Tmax: int, chain: int = 0) -> np.ndarray:
        """Planar loops W[R-1, T-1] = avg_wilson_loop((R,0,0), T) for R <= Rmax, T <= Tmax."""
        out = np.zeros((Rmax, Tmax))
        check(self._lib.mag_wilson_loops(self._h, chain, int(Rmax), int(Tmax), _dp(out)), "mag_wilson_loops")
        return out

    def check_constrained_plaquette(self, chain: int = 0) -> float:
        v = ctypes.c_double()
        check(self._lib.mag_constrained_plaquette(self._h, chain, ctypes.byref(v)), "mag_constrained_plaquette")
        return v.value

    # ------------------------------------------------------------ demon sweep
    def demon_microcanonical(self, n_sweeps: int, e_max: float, seed: int = 1, update_links: bool = False,
                             chain: int = 0) -> dict:
        """demon_microcanonical (field-demon.h:25-126): per-link demon sweeps with plaquette,
        rectangle, chair and twist demons.  Returns the demon energies after each sweep
        ([n_sweeps, 4]), the accepted / rejected hit counts and the reunitarisation deviation
        of each sweep."""
        E = np.zeros((int(n_sweeps), 4))
        dev = np.zeros(int(n_sweeps))
        a, r = ctypes.c_int64(), ctypes.c_int64()
        check(self._lib.mag_demon_microcanonical(self._h, chain, int(n_sweeps), float(e_max), int(seed),
                                                 1 if update_links else 0, _dp(E), ctypes.byref(a),
                                                 ctypes.byref(r), _dp(dev)), "mag_demon_microcanonical")
        return {"demon_energy": E, "accepted": a.value, "rejected": r.value, "reunit_maxdev": dev}

    def demon_microcanonical_all(self, n_sweeps: int, e_max: float, seed: int = 1,
                                 update_links: bool = False) -> list[dict]:
        """The per-link demon sweeps of every chain at once (one CTA per chain).  Chain c draws
        with the key seed + its stream index, so entry c equals
        demon_microcanonical(n_sweeps, e_max, seed + index, chain=c)."""
        n = self.n_chains
        E = np.zeros((n, int(n_sweeps), 4))
        dev = np.zeros((n, int(n_sweeps)))
        a, r = np.zeros(n, np.int64), np.zeros(n, np.int64)
        check(self._lib.mag_demon_microcanonical_all(self._h, int(n_sweeps), float(e_max), int(seed),
                                                     1 if update_links else 0, _dp(E),
                                                     a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                                     r.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _dp(dev)),
              "mag_demon_microcanonical_all")
        return [{"demon_energy": E[c], "accepted": int(a[c]), "rejected": int(r[c]), "reunit_maxdev": dev[c]}
                for c in range(n)]

    # ------------------------------------------------------------ NERSC I/O
    def export_config_nersc(self, path: str, beta: float | None = None, sequence_num: int = 0,
                            ensemble_label: str = "", skip_third: bool = True, chain: int = 0) -> dict:
        """export_config_nersc (field-matrix.h:452-572) with Arg_export (beta,
        sequence_num, ensemble_label); skip_third = doesSkipThird (DATATYPE
        4D_SU3_GAUGE).  Returns the header fields written and the digests."""
        info = _lib.NerscInfo()
        b = self.params[chain].beta if beta is None else float(beta)
        check(self._lib.mag_gauge_save_nersc(self._h, chain, str(path).encode(), 1 if skip_third else 0, b,
                                             int(sequence_num), ensemble_label.encode(), ctypes.byref(info)),
              "mag_gauge_save_nersc")
        return info.as_dict()

    def import_config_nersc(self, path: str, chain: int = 0) -> dict:
        """import_config_nersc (field-matrix.h:594-713).  Raises MagError with
        code MAG_ERR_FORMAT / MAG_ERR_CHECKSUM / MAG_ERR_PLAQUETTE / MAG_ERR_IO
        where the reference asserts."""
        info = _lib.NerscInfo()
        check(self._lib.mag_gauge_load_nersc(self._h, chain, str(path).encode(), ctypes.byref(info)),
              "mag_gauge_load_nersc")
        return info.as_dict()

    # ------------------------------------------------------------ timing
    def last_run_ms(self) -> float:
        v = ctypes.c_double()
        check(self._lib.mag_last_run_ms(self._h, ctypes.byref(v)), "mag_last_run_ms")
        return v.value

    def last_measure_ms(self) -> float:
        v = ctypes.c_double()
        check(self._lib.mag_last_measure_ms(self._h, ctypes.byref(v)), "mag_last_measure_ms")
        return v.value

    def time_force(self, reps: int) -> float:
        v = ctypes.c_double()
        check(self._lib.mag_time_force(self._h, int(reps), ctypes.byref(v)), "mag_time_force")
        return v.value

    def time_kernel(self, which: str, reps: int) -> float:
        v = ctypes.c_double()
        check(self._lib.mag_time_kernel(self._h, which.encode(), int(reps), ctypes.byref(v)), "mag_time_kernel")
        return v.value

    def autotune(self, reps: int = 3) -> dict:
        """Re-run the launch-configuration tuner; returns
        {family: {"fp64": [chosen variant, {variant: ms}], "fp32": [...]}}."""
        import json

        buf = ctypes.create_string_buffer(16384)
        check(self._lib.mag_autotune(self._h, int(reps), buf, len(buf)), "mag_autotune")
        return json.loads(buf.value.decode())

    def set_kernel_variant(self, family: str, precision: str, variant: str) -> None:
        """Use `variant` (e.g. "t1m3", "s6r128") for `family` at "fp64" or "fp32" in place of the tuner's choice."""
        check(self._lib.mag_set_kernel_variant(self._h, family.encode(), 0 if precision == "fp64" else 1,
                                               variant.encode()), "mag_set_kernel_variant")

    def graph_kernel_count(self) -> int:
        v = ctypes.c_int()
        check(self._lib.mag_graph_kernel_count(self._h, ctypes.byref(v)), "mag_graph_kernel_count")
        return v.value


def _matrices(a) -> np.ndarray:
    a = np.ascontiguousarray(a, np.complex128)
    assert a.shape[-2:] == (3, 3)
    return a


def expiq(Q) -> np.ndarray:
    """expiQ (field-hmc.h:82-123) of Hermitian traceless matrices Q[..., 3, 3] on the GPU."""
    q = _matrices(Q)
    out = np.empty_like(q)
    check(_lib.load().mag_expiq(_dp(q), q.size // 9, _dp(out)), "mag_expiq")
    return out


def dexpiq(Q, DQ) -> np.ndarray:
    """DexpiQ (field-multi.h:90-178): derivative of exp(iQ) at Q[..., 3, 3] along DQ, on the GPU."""
    q, d = _matrices(Q), _matrices(DQ)
    assert q.shape == d.shape
    out = np.empty_like(q)
    check(_lib.load().mag_dexpiq(_dp(q), _dp(d), q.size // 9, _dp(out)), "mag_dexpiq")
    return out


def compute_lambda(Q, SigmaP, U) -> np.ndarray:
    """compute_Lambda (field-multi.h:180-269) of triples (Q, Sigma', U)[..., 3, 3] on the GPU."""
    q, s, u = _matrices(Q), _matrices(SigmaP), _matrices(U)
    assert q.shape == s.shape == u.shape
    out = np.empty_like(q)
    check(_lib.load().mag_compute_lambda(_dp(q), _dp(s), _dp(u), q.size // 9, _dp(out)), "mag_compute_lambda")
    return out


def probe_fma_peak(precision: str = "fp64") -> float:
    """Measured CUDA-core FMA throughput of the current device (TFLOP/s, 2 flops per FMA)."""
    v = ctypes.c_double()
    code = {"fp64": 0, "fp32": 1, "fp32x2": 2, "fp32x2_selected": 3}[precision]
    check(_lib.load().mag_probe_fma_peak(code, ctypes.byref(v)), "mag_probe_fma_peak")
    return v.value


def read_nersc_header(path: str) -> dict:
    """The NERSC header fields of a file (no device work)."""
    info = _lib.NerscInfo()
    check(_lib.load().mag_nersc_read_header(str(path).encode(), ctypes.byref(info)), "mag_nersc_read_header")
    return info.as_dict()


def crc32_segmented(data: bytes, seg: int = 16384) -> int:
    """CRC-32 of ``data`` by the segment-and-chain scheme of the NERSC kernels (host)."""
    v = ctypes.c_uint32()
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    check(_lib.load().mag_crc32_host(buf, len(data), int(seg), ctypes.byref(v)), "mag_crc32_host")
    return v.value
