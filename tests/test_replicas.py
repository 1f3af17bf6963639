"""The multi-rank host logic of bench.py (replicas only: each rank runs its
own grid; the job time is the slowest rank's) on world_size-2 gloo groups."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 100.0 + 50.0 * rank  # rank 1 is slower
        m = bench.max_over_ranks(ms, world, "cpu")
        q.put((rank, m, bench.replica_throughput(world, 24, m)))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, m, v in res:
        assert m == pytest.approx(150.0)
        assert v == pytest.approx(2 * 24 * 1000.0 / 150.0)


def test_single_rank_is_identity():
    assert bench.max_over_ranks(12.5, 1, "cpu") == 12.5
    assert bench.replica_throughput(1, 10, 100.0) == pytest.approx(100.0)
