"""mag_b200 -- B200 (sm_100a) constrained SU(3) hybrid Monte Carlo.

A from-scratch implementation of the hot path of hummingtree/mag (Iwasaki
staples and gauge force, multi-level stout smearing and its derivative, the
force-gradient integrator with constrained link updates, Metropolis / demon
accept, compensated Hamiltonian sums, Wilson loops) as hand-written CUDA
kernels in libmag_b200.so behind the C ABI of include/mag_c.h.  ``Chmc``
mirrors the reference's field-*.h function names.
"""
from ._lib import MagError, load
from .field_hmc import Chmc, make_params, volume

__all__ = ["Chmc", "MagError", "load", "make_params", "volume"]
