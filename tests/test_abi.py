"""CPU checks of the drop-in boundary: the C-ABI library loads and exports
every entry point that include/*.h declares (no compute call without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from mag_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\s*\*?\s*(mag_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("mag_ctx_create", "mag_gauge_force", "mag_trajectory", "mag_run", "mag_wilson_loops",
                 "mag_stout_level", "mag_evolve_gauge", "mag_hamiltonian"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_library_is_built_for_sm100a():
    # the fatbin section names the target; check the build log recorded by mag_b200.build
    logs = glob.glob(os.path.join(ROOT, "mag_b200", "_build", "*.log"))
    if not logs:
        pytest.skip("no build logs in this checkout")
    for lg in logs:
        assert "arch=compute_100a,code=sm_100a" in open(lg).read().splitlines()[0]


def test_error_path_without_gpu_is_an_error_code():
    # creating a context needs a device; on a CPU box it must fail with a
    # status code and a message, never crash or fall back to the CPU
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    lib = _lib.load()
    from mag_b200.field_hmc import make_params
    p = make_params((4, 4, 4, 4))
    h = ctypes.c_void_p()
    rc = lib.mag_ctx_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == _lib.MAG_ERR_CUDA or rc == _lib.MAG_ERR_NOMEM
    assert lib.mag_last_error()


def test_invalid_params_are_rejected_before_any_device_work():
    lib = _lib.load()
    from mag_b200.field_hmc import make_params
    h = ctypes.c_void_p()
    bad = make_params((4, 4, 4, 4), mag=1)  # mag = 1 freezes every link
    assert lib.mag_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.MAG_ERR_ARG
    bad = make_params((4, 4, 3, 4), mag=2)  # extent not divisible by mag
    assert lib.mag_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.MAG_ERR_ARG
    assert lib.mag_ctx_create(None, ctypes.byref(h)) == _lib.MAG_ERR_ARG


def test_oracle_exports():
    import oracle
    lib = oracle.lib()
    for n in ("mo_force", "mo_trajectory", "mo_stout_forward", "mo_wilson_loop", "mo_constrained_plaquette"):
        assert hasattr(lib, n)
