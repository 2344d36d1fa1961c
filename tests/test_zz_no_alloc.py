"""The allocation-free entry point against the regular one.

mag_action_sums_noalloc is for callers that cannot call cudaMalloc (they pass
links and result slots that already live in device memory they manage).  This
test supplies those device buffers itself, calls the entry point twice in a
row on the same stream, and checks both results against mag_action (the
context-based entry point) at the tolerance used for action parity, 1e-12
relative.  It is collected last so that a stop-at-first-failure run has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_action_sums_noalloc_matches_mag_action():
    import torch

    import mag_b200 as M
    import oracle as O
    from mag_b200 import _lib

    dims = (8, 8, 8, 12)
    U = O.gen_hot(dims, 23)
    with M.Chmc(dims, mag=0, action="iwasaki") as c:
        c.set_gauge(U)
        plaq_ref, rect_ref, _ = c.gauge_action()

    lib = _lib.load()
    d_links = torch.from_numpy(np.ascontiguousarray(U).view(np.float64).reshape(-1)).to("cuda")
    d_sums = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    dims_c = (ctypes.c_int * 4)(*dims)
    torch.cuda.synchronize()
    for call in range(2):
        rc = lib.mag_action_sums_noalloc(dims_c, ctypes.c_void_p(d_links.data_ptr()),
                                         ctypes.c_void_p(d_sums.data_ptr()), None)
        assert rc == _lib.MAG_OK, lib.mag_last_error()
        torch.cuda.synchronize()
        plaq, rect = d_sums.tolist()
        assert abs(plaq - plaq_ref) <= 1e-12 * abs(plaq_ref), (call, plaq, plaq_ref)
        assert abs(rect - rect_ref) <= 1e-12 * abs(rect_ref), (call, rect, rect_ref)

    # a lattice beyond the static scratch is refused before any work
    big = (ctypes.c_int * 4)(256, 256, 256, 2)
    rc = lib.mag_action_sums_noalloc(big, ctypes.c_void_p(d_links.data_ptr()), ctypes.c_void_p(d_sums.data_ptr()),
                                     None)
    assert rc == _lib.MAG_ERR_ARG
    assert b"limit" in lib.mag_last_error()
