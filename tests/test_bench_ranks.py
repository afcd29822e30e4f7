"""Multi-rank aggregation of bench.py on CPU: two gloo ranks (one process each, as
torchrun would start them on two GPUs).  The time is the slowest rank's, the value
counts every rank's particles."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.over_ranks([1.0 + rank, 7.0 - rank], "max", dist, device="cpu")
        n = bench.over_ranks([1000 * (rank + 1)], "sum", dist, device="cpu")[0]
        out[rank] = (t, n, bench.job_rate(n, 5, t[0]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_all_particles():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        t, n, v = res[r]
        assert t == [2.0, 7.0]  # elementwise max over the two ranks
        assert n == 3000.0  # particles of both ranks
        assert v == pytest.approx(3000.0 * 5 / 2.0)


def test_single_process_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.over_ranks([3.0, 4.0], "max") == [3.0, 4.0]
    assert bench.job_rate(10, 3, 2.0) == 15.0
