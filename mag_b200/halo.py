"""Halo exchange between processes for a lattice split along x3 (one slab per process).

``TorchHaloExchange`` is a ``mag_halo_fn`` (include/mag_c.h) built on torch.distributed:
the role qlat's fetch_expanded_chart plays through MPI in the reference
(field-hmc.h:544-558) and its MPI_Allreduce of the Hamiltonian's sums (:628).

* ``MAG_HALO_EXCHANGE``: in each of the field's planes, the slab's lowest ``halo``
  interior time slices go to the lower neighbour (rank - 1) and its highest to the
  upper one (rank + 1); the neighbours' slices come back into the two halos.  With
  NCCL the transfers are device send/recv issued on the context's stream (so they
  are ordered after the kernels that produced the field and before those that read
  the halo); with gloo (CPU transport) the slices go through host copies after the
  stream has been synchronised.
* ``MAG_HALO_SUM``: all-reduce (sum) of the sums and (max) of the reunitarisation
  deviation.

Sends go in the order (to the lower neighbour, to the upper), receives in the order
(from the upper, from the lower), so that with two slabs, where both neighbours are
the same process, the i-th send of one side meets the i-th receive of the other.

``ShardChmc`` is the ``Chmc`` of one slab (mag_shard_create + mag_set_halo_fn).
"""
from __future__ import annotations

import ctypes
import sys
import traceback

import numpy as np

from . import _lib
from ._lib import MagParams, check
from .field_hmc import Chmc, make_params, volume

MAG_HALO_EXCHANGE, MAG_HALO_SUM = 0, 1


class HaloOp(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("rank", ctypes.c_int),
        ("nshards", ctypes.c_int),
        ("base", ctypes.c_void_p),
        ("nplanes", ctypes.c_int),
        ("plane_bytes", ctypes.c_size_t),
        ("slab_bytes", ctypes.c_size_t),
        ("send_lo", ctypes.c_size_t),
        ("send_hi", ctypes.c_size_t),
        ("recv_lo", ctypes.c_size_t),
        ("recv_hi", ctypes.c_size_t),
        ("sums", ctypes.POINTER(ctypes.c_double)),
        ("nsums", ctypes.c_int),
        ("maxval", ctypes.POINTER(ctypes.c_double)),
        ("stream", ctypes.c_void_p),
    ]


HALO_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(HaloOp))


class _DeviceBytes:
    """A device byte range as an object torch.as_tensor understands (__cuda_array_interface__)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def field_bytes(op: HaloOp, device: bool):
    """The whole field of an exchange as a flat uint8 tensor (device memory) or numpy array (host memory)."""
    n = op.nplanes * op.plane_bytes
    if device:
        import torch

        return torch.as_tensor(_DeviceBytes(op.base, n), device="cuda")
    return np.ctypeslib.as_array((ctypes.c_uint8 * n).from_address(op.base))


def exchange_plan(op: HaloOp):
    """[(plane, send offset, peer, tag)] and [(plane, receive offset, peer, tag)] in the issue order."""
    lo, hi = (op.rank - 1) % op.nshards, (op.rank + 1) % op.nshards
    sends, recvs = [], []
    for p in range(op.nplanes):
        base = p * op.plane_bytes
        sends.append((base + op.send_lo, lo, 2 * p))      # my lowest slices -> the lower neighbour's high halo
        sends.append((base + op.send_hi, hi, 2 * p + 1))  # my highest slices -> the upper neighbour's low halo
        recvs.append((base + op.recv_hi, hi, 2 * p))      # the upper neighbour's lowest slices
        recvs.append((base + op.recv_lo, lo, 2 * p + 1))  # the lower neighbour's highest slices
    return sends, recvs


class TorchHaloExchange:
    """mag_halo_fn over a torch.distributed process group (NCCL: device transfers on the
    context's stream; gloo: host staging).  ``device=False`` treats ``base`` as host memory
    (testing the plan on CPU ranks)."""

    def __init__(self, group=None, device: bool = True):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.device = device
        self.nccl = device and dist.get_backend(group) == "nccl"
        self.fn = HALO_FN(self._call)  # kept alive with this object

    def _call(self, user, op_ptr) -> int:
        try:
            op = op_ptr.contents
            if op.kind == MAG_HALO_SUM:
                self.sum(op)
            else:
                self.exchange(op)
            return 0
        except Exception:  # the library turns a non-zero status into MAG_ERR_STATE
            traceback.print_exc(file=sys.stderr)
            return 1

    def sum(self, op: HaloOp) -> None:
        import torch

        dist = self.dist
        dev = "cuda" if self.nccl else "cpu"
        t = torch.tensor([op.sums[i] for i in range(op.nsums)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        for i, v in enumerate(t.cpu().tolist()):
            op.sums[i] = v
        if op.maxval:
            m = torch.tensor([op.maxval[0]], dtype=torch.float64, device=dev)
            dist.all_reduce(m, op=dist.ReduceOp.MAX, group=self.group)
            op.maxval[0] = float(m.item())

    def exchange(self, op: HaloOp) -> None:
        import torch

        dist = self.dist
        sends, recvs = exchange_plan(op)
        n = op.slab_bytes
        if self.nccl:
            field = field_bytes(op, True)
            with torch.cuda.stream(torch.cuda.ExternalStream(op.stream)):
                ops = [dist.P2POp(dist.isend, field[o:o + n], peer, self.group, tag) for o, peer, tag in sends]
                ops += [dist.P2POp(dist.irecv, field[o:o + n], peer, self.group, tag) for o, peer, tag in recvs]
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            return
        if self.device:
            torch.cuda.ExternalStream(op.stream).synchronize()
            field = field_bytes(op, True)
            host_send = [field[o:o + n].cpu() for o, _, _ in sends]
        else:
            field = field_bytes(op, False)
            host_send = [torch.from_numpy(field[o:o + n].copy()) for o, _, _ in sends]
        host_recv = [torch.empty(n, dtype=torch.uint8) for _ in recvs]
        reqs = [dist.isend(b, peer, self.group, tag) for b, (_, peer, tag) in zip(host_send, sends)]
        reqs += [dist.irecv(b, peer, self.group, tag) for b, (_, peer, tag) in zip(host_recv, recvs)]
        for r in reqs:
            r.wait()
        for b, (o, _, _) in zip(host_recv, recvs):
            if self.device:
                field[o:o + n].copy_(b.to("cuda"))
            else:
                field[o:o + n] = b.numpy()
        if self.device:
            torch.cuda.synchronize()


def slab_dims(dims, nshards: int, halo: int):
    return (dims[0], dims[1], dims[2], dims[3] // nshards + 2 * halo)


def slab_of(field: np.ndarray, dims, nshards: int, rank: int, halo: int) -> np.ndarray:
    """The slab layout of rank `rank` (its slices plus `halo` slices of each neighbour) of a lattice field."""
    S3 = dims[0] * dims[1] * dims[2]
    loc = dims[3] // nshards
    t = (np.arange(loc + 2 * halo) + rank * loc - halo) % dims[3]
    return np.ascontiguousarray(field.reshape((dims[3], S3) + field.shape[1:])[t].reshape((-1,) + field.shape[1:]))


def interior_of(slab: np.ndarray, dims, nshards: int, halo: int) -> np.ndarray:
    """The slab's own time slices (a lattice field's slices [rank, rank + 1) dims[3] / nshards)."""
    S3 = dims[0] * dims[1] * dims[2]
    return slab[halo * S3:(halo + dims[3] // nshards) * S3]


class ShardChmc(Chmc):
    """Chmc of slab `rank` of a lattice split along x3 into `nshards` slabs with `halo` slices
    of each neighbour; fields are in the slab's layout (``slab_of``)."""

    def __init__(self, dims, nshards: int, rank: int, halo: int = 2, exchange: TorchHaloExchange | None = None,
                 **kw):
        self._lib = _lib.load()
        p = make_params(dims, **kw)
        h = ctypes.c_void_p()
        check(self._lib.mag_shard_create(ctypes.byref(p), int(nshards), int(rank), int(halo), ctypes.byref(h)),
              "mag_shard_create")
        self._h = h
        self.params = [p]
        self.lattice_dims = tuple(dims)
        self.dims = [slab_dims(dims, nshards, halo)]
        self.n_chains = 1
        self.nshards, self.rank, self.halo = nshards, rank, halo
        self.exchange = exchange
        if exchange is not None:
            check(self._lib.mag_set_halo_fn(self._h, ctypes.cast(exchange.fn, ctypes.c_void_p), None), "mag_set_halo_fn")


__all__ = ["HaloOp", "ShardChmc", "TorchHaloExchange", "exchange_plan", "interior_of", "slab_of", "slab_dims"]
