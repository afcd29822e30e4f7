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


def test_roofline_numerators():
    """The algorithmic bytes bench.py divides by kernel time: the owner PM3 deposit writes
    every cell of every class-2 box once as float and reads each position code once; the
    PM3 FFT passes move the float mesh and the half spectrum once each way."""
    sys.path.insert(0, ROOT)
    import bench
    from cube_nu_b200.params import config_512

    p = config_512()
    n = p.npglobal
    napm = [0, 0, p.ns3, 0, 0, 0]
    nft = p.nft(2)
    assert bench.kernel_bytes(p, "deposit_pm3", n, napm, True) == p.ns3 * nft ** 3 * 4 + n * 3 * p.izipx
    nh = nft * nft * (nft // 2 + 1) * p.ns3
    assert bench.kernel_bytes(p, "fft_x_pm3", n, napm, True) == p.ns3 * nft ** 3 * 4 + nh * 8
    assert bench.kernel_bytes(p, "fft_c2r_pm3", n, napm, True) == nh * 8 + p.ns3 * nft ** 3 * 4
    assert bench.kernel_bytes(p, "fft_y_pm3", n, napm, True) == 2 * 2 * nh * 8
    for name in ("deposit_pm1", "deposit_pm2", "interp_pm1", "interp_pm2", "interp_pm3", "pp", "drift_dest",
                 "drift_gather", "fft_x_pm2", "fft_z_green_pm3"):
        b = bench.kernel_bytes(p, name, n, napm, True)
        assert isinstance(b, int) and b > 0, name
    assert bench.kernel_bytes(p, "momentum", n, napm, True) is None
    assert bench.job_rate(4 * n, 20, 2.0) == 4 * n * 10
