"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1).

With N GPUs every rank advances its own replica; the only collective is the
max over ranks of the device time.  This checks that reduction, that the
replicas get distinct seeds and identical workload parameters, and that the
ranks take the same collective steps.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        per_rank_ms = [12.5, 17.25][rank]
        m = bench.max_over_ranks(per_rank_ms, dist, "cpu")
        p = bench.workload_params("ensemble_96chains")
        q.put((rank, m, bench.rank_seed(rank), p["chains"][7]["beta"], bench.total_sites(p)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_timing_and_keep_replicas_distinct():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[1] for r in res] == [17.25, 17.25]          # max over ranks on every rank
    assert res[0][2] != res[1][2]                          # replica seeds differ
    assert res[0][3] == res[1][3] and res[0][4] == res[1][4]  # same workload on every rank
    assert res[0][4] == 48 * 8 ** 4 + 32 * 12 ** 4 + 16 * 16 ** 4


def test_single_process_needs_no_group():
    import bench

    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0


def test_partition_balances_the_ensemble():
    import bench
    from mag_b200.ensemble import chain_cost, imbalance, partition

    chains = bench.workload_params("ensemble_96chains")["chains"]
    costs = [chain_cost(c["dims"], 8) for c in chains]
    for world in (1, 2, 3, 4, 8):
        parts = partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(chains)))                     # every chain exactly once
        assert parts == partition(costs, world)                     # the same split on every rank
        assert imbalance(costs, parts) < 1.0 + max(costs) / (sum(costs) / world)  # LPT bound
    assert imbalance(costs, partition(costs, 2)) < 1.01
    assert imbalance(costs, partition(costs, 8)) < 1.1


def _gather_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from mag_b200.ensemble import gather_records, partition

        costs = [5, 1, 4, 2, 3, 3, 1]
        parts = partition(costs, world)
        # trajectory t of global chain c: delta_h = 100 t + c, accept = c % 2
        recs = [[{"delta_h": 100.0 * t + c, "accept": c % 2, "avg_plaquette": 0.5 + c, "h_old": 1.0, "h_new": 2.0,
                  "uniform": 0.25, "reunit_maxdev": 0.0} for c in parts[rank]] for t in range(3)]
        out = gather_records(recs, parts, rank, dist, "cpu")
        q.put((rank, [[(r["delta_h"], r["accept"]) for r in row] for row in out], parts))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gather_records_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    expect = [[(100.0 * t + c, c % 2) for c in range(7)] for t in range(3)]
    assert res[0][1] == expect and res[1][1] == expect
    assert res[0][2][0] and res[0][2][1]   # both ranks hold chains



def _halo_worker(rank, world, port, q, dims, halo):
    """One slab per gloo rank, in host memory laid out as the library lays out a shard's field:
    4 planes of the slab's (dims[3] / world + 2 halo) time slices, planes padded apart."""
    import ctypes
    import datetime

    import numpy as np
    import torch.distributed as dist

    from mag_b200.halo import HaloOp, MAG_HALO_EXCHANGE, MAG_HALO_SUM, TorchHaloExchange

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        S3, unit = dims[0] * dims[1] * dims[2], 24          # bytes per site and plane (three int64)
        L3, loc = dims[3], dims[3] // world
        ext = loc + 2 * halo
        per_plane = ext * S3 * 3 + 40                       # int64 words, a gap between planes
        lattice = np.arange(4 * L3 * S3 * 3, dtype=np.int64).reshape(4, L3, S3 * 3)
        field = np.full((4, per_plane), -1, dtype=np.int64)
        t = (np.arange(ext) + rank * loc - halo) % L3
        for p in range(4):
            field[p, halo * S3 * 3:(halo + loc) * S3 * 3] = lattice[p, t[halo:halo + loc]].reshape(-1)
        op = HaloOp()
        op.kind, op.rank, op.nshards, op.nplanes = MAG_HALO_EXCHANGE, rank, world, 4
        op.base = field.ctypes.data
        op.plane_bytes = per_plane * 8
        op.slab_bytes = halo * S3 * unit
        op.send_lo, op.send_hi = halo * S3 * unit, loc * S3 * unit
        op.recv_lo, op.recv_hi = 0, (halo + loc) * S3 * unit
        ex = TorchHaloExchange(device=False)
        assert ex._call(None, ctypes.pointer(op)) == 0
        ok = all(np.array_equal(field[p, :ext * S3 * 3], lattice[p, t].reshape(-1)) for p in range(4))
        ok = ok and np.all(field[:, ext * S3 * 3:] == -1)   # nothing written into the gaps
        # the Hamiltonian's sums and the reunitarisation maximum over the slabs
        sums = (ctypes.c_double * 2)(1.5 * (rank + 1), 1e-17)
        mx = ctypes.c_double(0.25 * rank)
        sop = HaloOp()
        sop.kind, sop.rank, sop.nshards = MAG_HALO_SUM, rank, world
        sop.sums, sop.nsums, sop.maxval = sums, 2, ctypes.pointer(mx)
        assert ex._call(None, ctypes.pointer(sop)) == 0
        q.put((rank, ok, sums[0], sums[1], mx.value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims,halo", [(2, (4, 2, 2, 8), 2), (3, (2, 2, 2, 12), 2), (2, (2, 2, 4, 8), 3)])
def test_gloo_halo_exchange_fills_every_slab_halo(world, dims, halo):
    """The halo exchange a process-per-slab run does through torch.distributed (mag_b200.halo),
    on CPU ranks with host buffers: every halo slice equals the lattice's, plane by plane, for
    two slabs (both neighbours the same rank) and three; the sums and the maximum reduce."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_halo_worker, args=(r, world, port, q, dims, halo)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(r[1] for r in res)
    total = sum(1.5 * (r + 1) for r in range(world))
    assert all(r[2] == total and abs(r[3] - world * 1e-17) < 1e-30 and r[4] == 0.25 * (world - 1) for r in res)
