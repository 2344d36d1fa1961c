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
