"""ctypes binding of libmag_b200.so (the C ABI declared in include/mag_c.h).

The library is the only compute path: if it is missing or cannot be loaded
this module raises, and nothing falls back to a CPU implementation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmag_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "mag_c.h")

MAG_OK = 0
MAG_ERR_ARG = -1
MAG_ERR_CUDA = -2
MAG_ERR_NAN = -3
MAG_ERR_STATE = -4
MAG_ERR_NOMEM = -5
MAG_ERR_IO = -6
MAG_ERR_FORMAT = -7
MAG_ERR_CHECKSUM = -8
MAG_ERR_PLAQUETTE = -9

ACTION_WILSON, ACTION_IWASAKI = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
INT_FORCE_GRADIENT, INT_LEAPFROG = 0, 1
ACCEPT_METROPOLIS, ACCEPT_DEMON = 0, 1


class MagParams(ctypes.Structure):
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
        ("precision", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("accept", ctypes.c_int),
        ("e_max", ctypes.c_double),
        ("n_forced_accept", ctypes.c_int),
        ("seed", ctypes.c_uint64),
    ]


class TrajResult(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "h_old", "h_new", "delta_h", "kinetic_old", "kinetic_new", "action_old", "action_new",
        "plaq_sum_old", "plaq_sum_new", "rect_sum_old", "rect_sum_new", "uniform")] + [
        ("demon", ctypes.c_double * 2),
        ("reunit_maxdev", ctypes.c_double),
        ("avg_plaquette", ctypes.c_double),
        ("accept", ctypes.c_int),
        ("traj", ctypes.c_int),
    ]

    def as_dict(self) -> dict:
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["demon"] = [self.demon[0], self.demon[1]]
        return d


class NerscInfo(ctypes.Structure):
    """mag_nersc_info: NERSC header fields and the digests computed from the payload."""

    _fields_ = [
        ("dims", ctypes.c_int * 4),
        ("two_row", ctypes.c_int),
        ("payload_offset", ctypes.c_int64),
        ("checksum_header", ctypes.c_uint32),
        ("checksum", ctypes.c_uint32),
        ("crc32_header", ctypes.c_uint32),
        ("crc32", ctypes.c_uint32),
        ("plaquette_header", ctypes.c_double),
        ("plaquette", ctypes.c_double),
        ("link_trace_header", ctypes.c_double),
        ("link_trace", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["dims"] = list(self.dims)
        return d


class MagError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


_DP = ctypes.POINTER(ctypes.c_double)
_CTX = ctypes.c_void_p
_IP = ctypes.POINTER(ctypes.c_int)

# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "mag_ctx_create": [ctypes.POINTER(MagParams), ctypes.POINTER(_CTX)],
    "mag_ensemble_create": [ctypes.POINTER(MagParams), ctypes.c_int, ctypes.POINTER(_CTX)],
    "mag_ctx_destroy": [_CTX],
    "mag_last_error": [],
    "mag_ctx_num_chains": [_CTX, _IP],
    "mag_ctx_device_bytes": [_CTX, ctypes.POINTER(ctypes.c_size_t)],
    "mag_gauge_set": [_CTX, ctypes.c_int, _DP],
    "mag_gauge_get": [_CTX, ctypes.c_int, _DP],
    "mag_gauge_hot_start": [_CTX, ctypes.c_uint64],
    "mag_gauge_cold_start": [_CTX],
    "mag_momentum_set": [_CTX, ctypes.c_int, _DP],
    "mag_momentum_get": [_CTX, ctypes.c_int, _DP],
    "mag_momentum_refresh": [_CTX, ctypes.c_uint64],
    "mag_uniforms_set": [_CTX, _DP],
    "mag_gauge_force": [_CTX, ctypes.c_int, _DP],
    "mag_staple": [_CTX, ctypes.c_int, _DP],
    "mag_action": [_CTX, ctypes.c_int, _DP, _DP, _DP],
    "mag_plaquette": [_CTX, ctypes.c_int, _DP],
    "mag_kinetic": [_CTX, ctypes.c_int, _DP],
    "mag_hamiltonian": [_CTX, ctypes.c_int, _DP],
    "mag_evolve_gauge": [_CTX, ctypes.c_double],
    "mag_evolve_momentum": [_CTX, ctypes.c_double],
    "mag_evolve_gauge_src": [_CTX, ctypes.c_double, ctypes.c_int],
    "mag_stout_forward": [_CTX, ctypes.c_int, ctypes.c_int, _DP],
    "mag_stout_force": [_CTX, ctypes.c_int, _DP],
    "mag_fg_trajectory": [_CTX, ctypes.c_int, ctypes.POINTER(TrajResult)],
    "mag_batch_create": [ctypes.POINTER(MagParams), ctypes.c_int, ctypes.POINTER(_CTX)],
    "mag_batch_run": [_CTX, ctypes.c_int, ctypes.POINTER(TrajResult)],
    "mag_set_stream_index": [_CTX, ctypes.POINTER(ctypes.c_int64)],
    "mag_demon_microcanonical": [_CTX, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_int,
                                 _DP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _DP],
    "mag_expiq": [_DP, ctypes.c_int64, _DP],
    "mag_compute_lambda": [_DP, _DP, _DP, ctypes.c_int64, _DP],
    "mag_dexpiq": [_DP, _DP, ctypes.c_int64, _DP],
    "mag_demon_microcanonical_all": [_CTX, ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_int, _DP,
                                     ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _DP],
    "mag_reunitarize": [_CTX, _DP],
    "mag_stout_level": [_CTX, ctypes.c_int, ctypes.c_int, _DP],
    "mag_integrate": [_CTX],
    "mag_trajectory": [_CTX, ctypes.c_int, ctypes.POINTER(TrajResult)],
    "mag_run": [_CTX, ctypes.c_int, ctypes.POINTER(TrajResult)],
    "mag_traj_counter": [_CTX, ctypes.POINTER(ctypes.c_int64)],
    "mag_set_traj_counter": [_CTX, ctypes.c_int64],
    "mag_wilson_loop": [_CTX, ctypes.c_int, _IP, ctypes.c_int, _DP],
    "mag_wilson_loops": [_CTX, ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP],
    "mag_constrained_plaquette": [_CTX, ctypes.c_int, _DP],
    "mag_last_run_ms": [_CTX, _DP],
    "mag_last_measure_ms": [_CTX, _DP],
    "mag_time_force": [_CTX, ctypes.c_int, _DP],
    "mag_time_kernel": [_CTX, ctypes.c_char_p, ctypes.c_int, _DP],
    "mag_graph_kernel_count": [_CTX, _IP],
    "mag_autotune": [_CTX, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t],
    "mag_set_kernel_variant": [_CTX, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p],
    "mag_action_sums_noalloc": [_IP, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    "mag_probe_fma_peak": [ctypes.c_int, _DP],
    "mag_gauge_load_nersc": [_CTX, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(NerscInfo)],
    "mag_gauge_save_nersc": [_CTX, ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                             ctypes.c_char_p, ctypes.POINTER(NerscInfo)],
    "mag_nersc_read_header": [ctypes.c_char_p, ctypes.POINTER(NerscInfo)],
    "mag_crc32_host": [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint32)],
    "mag_dd_create": [ctypes.POINTER(MagParams), ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "mag_dd_destroy": [ctypes.c_void_p],
    "mag_dd_gauge_set": [ctypes.c_void_p, _DP],
    "mag_dd_gauge_get": [ctypes.c_void_p, _DP],
    "mag_dd_momentum_set": [ctypes.c_void_p, _DP],
    "mag_dd_momentum_get": [ctypes.c_void_p, _DP],
    "mag_dd_hot_start": [ctypes.c_void_p, ctypes.c_uint64],
    "mag_dd_uniforms_set": [ctypes.c_void_p, _DP],
    "mag_dd_gauge_force": [ctypes.c_void_p, _DP],
    "mag_dd_trajectory": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(TrajResult)],
    "mag_dd_shard": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_CTX)],
    "mag_shard_create": [ctypes.POINTER(MagParams), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_CTX)],
    "mag_set_halo_fn": [_CTX, ctypes.c_void_p, ctypes.c_void_p],
    "mag_multi_create": [ctypes.POINTER(MagParams), ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)],
    "mag_multi_destroy": [ctypes.c_void_p],
    "mag_multi_gauge_set": [ctypes.c_void_p, _DP, _DP],
    "mag_multi_gauge_get": [ctypes.c_void_p, _DP, _DP],
    "mag_multi_momentum_set": [ctypes.c_void_p, _DP, _DP],
    "mag_multi_forces": [ctypes.c_void_p, _DP, _DP],
    "mag_multi_hamiltonian": [ctypes.c_void_p, _DP],
    "mag_multi_trajectory": [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _DP],
}
_RESTYPE = {"mag_last_error": ctypes.c_char_p}

_lib = None


def load() -> ctypes.CDLL:
    """Load libmag_b200.so (build it first with ``python -m mag_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m mag_b200.build` (nvcc, sm_100a)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = lib
    return _lib


def check(code: int, where: str) -> None:
    if code != MAG_OK:
        msg = load().mag_last_error()
        raise MagError(code, where, msg.decode() if msg else "")
