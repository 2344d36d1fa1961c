"""Domain decomposition along x3 (mag_dd_*): a lattice held as slabs with halos.

The reference splits a lattice over MPI ranks, each holding its slab in a qlat
Field with expanded Geometry (field-hmc.h:777-781) refreshed by
fetch_expanded_chart before every force (field-hmc.h:544-558), and adds the
Hamiltonian's sums with MPI_Allreduce (field-hmc.h:628).  Here the slabs are
contexts on one GPU whose halos are refreshed by device copies.  On the GPU:
the force of the split lattice equals the undivided context's link for link
(the same kernels see the same neighbour links) and the oracle's to 1e-11;
trajectories from host momenta and uniforms give the undivided context's
Delta H (sums added over slabs in another order: 1e-10), accept bits and links;
the device Philox hot start and momenta use whole-lattice site indices, so a
split run with refreshed momenta repeats the undivided run.  On the CPU: the
arguments the split needs are checked before any device work.
"""
import ctypes

import numpy as np
import pytest

import mag_b200 as M
from mag_b200 import _lib
from mag_b200.field_hmc import make_params

DIMS = (8, 4, 4, 16)  # 128 sites per time slice (a multiple of the 32-site tile)
KW = dict(mag=2, action="iwasaki", beta=2.25, c1=-0.331, rho=0.1, n_stout=3, n_steps=6, tau=1.0)


@pytest.mark.parametrize("dims,nshards,halo,code", [
    ((8, 4, 4, 16), 3, 2, "divide"), ((8, 4, 4, 16), 16, 2, "halo depth"), ((8, 4, 4, 16), 2, 1, "halo depth"),
    ((8, 4, 4, 12), 4, 3, "multiple of mag"), ((6, 6, 6, 8), 2, 2, "multiple of 32")])
def test_split_arguments_are_checked_before_device_work(dims, nshards, halo, code):
    lib = _lib.load()
    p = make_params(dims, mag=2)
    h = ctypes.c_void_p()
    rc = lib.mag_dd_create(ctypes.byref(p), nshards, halo, ctypes.byref(h))
    assert rc == _lib.MAG_ERR_ARG
    assert code.encode() in lib.mag_last_error()
    assert not h.value


@pytest.mark.gpu
@pytest.mark.parametrize("nshards,halo,precision", [(1, 2, "fp64"), (2, 2, "fp64"), (4, 2, "fp64"), (2, 3, "fp64"),
                                                    (2, 2, "mixed")])
def test_split_force_equals_the_undivided_lattice(nshards, halo, precision):
    import oracle as O

    U = O.gen_hot(DIMS, 12)
    with M.Chmc(DIMS, precision=precision, **KW) as c:
        c.set_gauge(U)
        F1 = c.get_force()
    from mag_b200.dd import DomainChmc

    with DomainChmc(DIMS, nshards, halo, precision=precision, **KW) as d:
        d.set_gauge(U)
        assert np.array_equal(d.get_gauge(), U)
        Fd = d.get_force()
    assert np.abs(Fd - F1).max() <= 1e-14 * np.abs(F1).max()
    if precision == "fp64":
        po = O.make_params(DIMS, mag=2, action=1, beta=2.25, c1=-0.331, rho=0.1, n_stout=3)
        Fo = O.force(po, U)
        assert np.abs(Fd - Fo).max() / np.abs(Fo).max() < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("nshards", [2, 4])
def test_split_trajectories_equal_the_undivided_lattice(nshards):
    import oracle as O
    from mag_b200.dd import DomainChmc

    U = O.gen_hot(DIMS, 13)
    po = O.make_params(DIMS, mag=2, action=1, beta=2.25, c1=-0.331, rho=0.1, n_stout=3, n_steps=6)
    Uo = U.copy()
    with M.Chmc(DIMS, **KW) as c, DomainChmc(DIMS, nshards, 2, **KW) as d:
        c.set_gauge(U)
        d.set_gauge(U)
        for t in range(3):
            P = O.gen_momenta(DIMS, 5, t)
            u = O.gen_uniform(5, t)
            c.init_momentum(P)
            d.init_momentum(P)
            c.set_uniforms([u])
            d.set_uniforms([u])
            (r1,) = c.trajectory(refresh_momenta=False)
            rd = d.trajectory(refresh_momenta=False)
            assert rd["accept"] == r1["accept"]
            assert abs(rd["delta_h"] - r1["delta_h"]) < 1e-10, (rd["delta_h"], r1["delta_h"])
            assert abs(rd["h_old"] - r1["h_old"]) <= 1e-13 * abs(r1["h_old"])
            assert abs(rd["avg_plaquette"] - r1["avg_plaquette"]) < 1e-13
            assert rd["reunit_maxdev"] == r1["reunit_maxdev"]
            assert np.abs(d.get_gauge() - c.get_gauge()).max() < 1e-13
            if t == 0:
                Uo, o = O.trajectory(po, 0, Uo, P, u, [0.0, 0.0])
                assert abs(rd["delta_h"] - o["delta_h"]) < 1e-9
                assert rd["accept"] == o["accept"]


@pytest.mark.gpu
def test_split_device_rng_repeats_the_undivided_run():
    from mag_b200.dd import DomainChmc

    kw = dict(KW, n_stout=1, seed=17)
    with M.Chmc(DIMS, **kw) as c, DomainChmc(DIMS, 2, 2, **kw) as d:
        c.hot_start(4)
        d.hot_start(4)
        assert np.array_equal(d.get_gauge(), c.get_gauge())
        for _ in range(2):
            (r1,) = c.trajectory(refresh_momenta=True)
            rd = d.trajectory(refresh_momenta=True)
            assert rd["accept"] == r1["accept"] and abs(rd["delta_h"] - r1["delta_h"]) < 1e-10
        assert np.abs(d.get_gauge() - c.get_gauge()).max() < 1e-13


def _shard_proc(rank, world, port, q, halo):
    import datetime
    import os

    import torch
    import torch.distributed as dist

    import oracle as O
    from mag_b200.halo import ShardChmc, TorchHaloExchange, interior_of, slab_of

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        U = O.gen_hot(DIMS, 12)
        P = O.gen_momenta(DIMS, 5, 0)
        ex = TorchHaloExchange()
        with ShardChmc(DIMS, world, rank, halo, exchange=ex, **KW) as c:
            c.set_gauge(slab_of(U, DIMS, world, rank, halo))
            F = interior_of(c.get_force(), DIMS, world, halo)
            c.init_momentum(slab_of(P, DIMS, world, rank, halo))
            c.set_uniforms([O.gen_uniform(5, 0)])
            (r,) = c.trajectory(refresh_momenta=False)
            Ui = interior_of(c.get_gauge(), DIMS, world, halo)
        q.put((rank, F, r["delta_h"], r["accept"], r["h_old"], Ui))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_one_slab_per_process_through_the_halo_callback():
    """mag_shard_create + mag_set_halo_fn with mag_b200.halo.TorchHaloExchange: two processes on
    the one GPU, each holding one slab, exchanging halos and sums through gloo (host copies; no
    kernel waits on another process).  Force, Delta H, accept bit and links equal the undivided
    lattice's."""
    import socket

    import torch.multiprocessing as mp

    import oracle as O

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    world, halo = 2, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_proc, args=(r, world, port, q, halo)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    U = O.gen_hot(DIMS, 12)
    P = O.gen_momenta(DIMS, 5, 0)
    with M.Chmc(DIMS, **KW) as c:
        c.set_gauge(U)
        F1 = c.get_force()
        c.init_momentum(P)
        c.set_uniforms([O.gen_uniform(5, 0)])
        (r1,) = c.trajectory(refresh_momenta=False)
        U1 = c.get_gauge()
    F = np.concatenate([r[1] for r in res])
    assert np.abs(F - F1).max() <= 1e-14 * np.abs(F1).max()
    for r in res:
        assert r[3] == r1["accept"]
        assert abs(r[2] - r1["delta_h"]) < 1e-10
        assert abs(r[4] - r1["h_old"]) <= 1e-13 * abs(r1["h_old"])
    assert np.abs(np.concatenate([r[5] for r in res]) - U1).max() < 1e-13
