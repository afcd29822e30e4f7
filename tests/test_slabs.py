"""A run split into z-slabs over ranks, on the CPU: the slab geometry of cube_slab_cells
(host arithmetic of the library), the split and join of a whole-box state, and the
TorchComm collectives (cube_nu_b200/slabs.py) over gloo with two and three ranks, driven
through the C callback pointers the library calls.  The ghost-layer exchange is replayed
with the library's message order (sizes, counts, then particles) on a synthetic state,
and every rank's ghosts are checked against the whole box.  The device side (packing,
stepping) is covered by tests/test_gpu_slabs.py."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from cube_nu_b200 import slabs
from cube_nu_b200.params import Params
from tests.helpers import clustered_state

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _geom(nslab=2, slab=0, ng=128, nnt=4):
    return Params(ng=ng, nnt=nnt, nns=2, np_nc=2, izipx=1, nslab=nslab, slab=slab)


def _coords(p, cells):
    """Global coarse coordinates (N,3) of storage indices (inverse of cell_order)."""
    nt, nnt = p.nt, p.nnt
    c = np.asarray(cells)
    l = c % nt ** 3
    t = c // nt ** 3
    lx, ly, lz = l % nt, (l // nt) % nt, l // nt ** 2
    tx, ty, tz = t % nnt, (t // nnt) % nnt, t // nnt ** 2
    return np.stack([tx * nt + lx, ty * nt + ly, tz * nt + lz], axis=1)


@pytest.mark.parametrize("nslab,nnt", [(2, 2), (2, 4), (4, 4)])
def test_slab_cells_partition_and_layers(nslab, nnt):
    ng = 32 * nnt
    p0 = _geom(nslab, 0, ng=ng, nnt=nnt)
    own = [slabs.slab_cells(_geom(nslab, s, ng=ng, nnt=nnt), 0) for s in range(nslab)]
    allc = np.concatenate(own)
    assert np.array_equal(np.sort(allc), np.arange(p0.ncells))  # every cell owned once
    for s in range(nslab):
        p = _geom(nslab, s, ng=ng, nnt=nnt)
        c0, c1 = slabs.cell_range(p, nslab, s)
        assert np.array_equal(own[s], np.arange(c0, c1))
        z0, z1 = c0 // (p.nt ** 3 * p.nnt ** 2) * p.nt, c1 // (p.nt ** 3 * p.nnt ** 2) * p.nt  # cell layers [z0, z1)
        lay = {w: slabs.slab_cells(p, w) for w in (1, 2, 3, 4)}
        for w in lay:
            assert np.all(np.diff(lay[w]) > 0)  # ascending storage order
        z = {w: _coords(p, lay[w])[:, 2] for w in lay}
        assert set(z[1]) == set(range(z0, z0 + p.ncb))
        assert set(z[2]) == set(range(z1 - p.ncb, z1))
        assert set(z[3]) == {(z0 - k) % p.nc for k in range(1, p.ncb + 1)}
        assert set(z[4]) == {(z1 + k) % p.nc for k in range(p.ncb)}
        for w in lay:  # whole x-y planes
            assert len(lay[w]) == p.ncb * p.nc * p.nc
        # what this slab sends up is what the slab above takes as ghosts from below
        above = _geom(nslab, (s + 1) % nslab, ng=ng, nnt=nnt)
        below = _geom(nslab, (s - 1) % nslab, ng=ng, nnt=nnt)
        assert np.array_equal(lay[2], slabs.slab_cells(above, 3))
        assert np.array_equal(lay[1], slabs.slab_cells(below, 4))


def test_one_slab_has_no_layers():
    p = _geom(1, 0)
    assert len(slabs.slab_cells(p, 0)) == p.ncells
    for w in (1, 2, 3, 4):
        assert len(slabs.slab_cells(p, w)) == 0


def test_split_and_join_are_inverse():
    p = _geom()
    st = clustered_state(p, 40000, seed=3)
    parts = slabs.split_state(p, *st, 4)
    assert sum(q[0].shape[0] for q in parts) == st[0].shape[0]
    for s, q in enumerate(parts):
        c0, c1 = slabs.cell_range(p, 4, s)
        assert q[3][:c0].sum() == 0 and q[3][c1:].sum() == 0
        assert q[3].sum() == q[0].shape[0]
    back = slabs.join_states(parts)
    for a, b in zip(back, st):
        assert np.array_equal(a, b)


def test_params_reject_bad_slabs():
    with pytest.raises(ValueError):
        _geom(3, 0).validate()  # 3 does not divide nnt = 4
    with pytest.raises(ValueError):
        _geom(2, 2).validate()


# ---------------------------------------------------------------------------------
# gloo ranks
# ---------------------------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pack(st, start, cells):
    """Counts and particles (codes, velocities, ids) of `cells`, in that order."""
    xp, vp, pid, rhoc = st
    cnt = rhoc[cells].astype(np.int32)
    idx = np.concatenate([np.arange(start[c], start[c + 1]) for c in cells]) if len(cells) else np.zeros(0, int)
    return cnt, xp[idx], vp[idx], pid[idx]


def _payload(x, v, i):
    return np.concatenate([x.view(np.uint8).ravel(), v.view(np.uint8).ravel(), i.view(np.uint8).ravel()])


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from cube_nu_b200 import slabs as S

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        comm = S.TorchComm()
        cc = comm.as_c()
        res = {}
        # allreduce on host buffers, every dtype and both ops
        for dt, npt in ((S.DT_F32, np.float32), (S.DT_I64, np.int64), (S.DT_F64, np.float64), (S.DT_I32, np.int32)):
            a = (np.arange(5) * (rank + 1) + rank).astype(npt)
            rc = cc.allreduce(None, a.ctypes.data, a.size, dt, S.OP_SUM, 0)
            b = (np.arange(5) - 2 * rank).astype(npt)
            rc |= cc.allreduce(None, b.ctypes.data, b.size, dt, S.OP_MAX, 0)
            res["ar%d" % dt] = (rc, a.tolist(), b.tolist())
        # the ghost exchange of a whole-box state, in the library's message order
        p = Params(ng=64 * world, nnt=2 * world, nns=2, np_nc=2, izipx=1)
        st = clustered_state(p, 30000, seed=5)
        start = np.concatenate([[0], np.cumsum(st[3], dtype=np.int64)])
        ps = S.slab_params(p, world, rank)
        mine = S.split_state(p, *st, world)[rank]
        mstart = np.concatenate([[0], np.cumsum(mine[3], dtype=np.int64)])
        down = _pack(mine, mstart, S.slab_cells(ps, 1))
        up = _pack(mine, mstart, S.slab_cells(ps, 2))
        nout = np.array([up[0].sum(), down[0].sum()], dtype=np.int64)
        nin = np.zeros(2, dtype=np.int64)
        rc = cc.sendrecv(None, nout[0:].ctypes.data, 8, nout[1:].ctypes.data, 8, nin[0:].ctypes.data, 8,
                         nin[1:].ctypes.data, 8, 0)
        nlay = len(S.slab_cells(ps, 3))
        cin = [np.zeros(nlay, np.int32), np.zeros(nlay, np.int32)]
        rc |= cc.sendrecv(None, up[0].ctypes.data, 4 * nlay, down[0].ctypes.data, 4 * nlay, cin[0].ctypes.data,
                          4 * nlay, cin[1].ctypes.data, 4 * nlay, 0)
        pu, pd = _payload(*up[1:]), _payload(*down[1:])
        per = 3 * 1 + 12 + 8
        pin = [np.zeros(int(nin[0]) * per, np.uint8), np.zeros(int(nin[1]) * per, np.uint8)]
        rc |= cc.sendrecv(None, pu.ctypes.data, pu.size, pd.ctypes.data, pd.size, pin[0].ctypes.data, pin[0].size,
                          pin[1].ctypes.data, pin[1].size, 0)
        ok = rc == 0 and not comm.errors
        for k, which in ((0, 3), (1, 4)):  # ghosts from below, from above: the whole box's cells
            ref = _pack(st, start, S.slab_cells(ps, which))
            n = int(nin[k])
            ok &= np.array_equal(cin[k], ref[0]) and n == ref[0].sum()
            b = pin[k]
            ok &= np.array_equal(b[:3 * n].view(np.int8).reshape(n, 3), ref[1])
            ok &= np.array_equal(b[3 * n:15 * n].view(np.float32).reshape(n, 3), ref[2])
            ok &= np.array_equal(b[15 * n:].view(np.int64), ref[3])
        res["exchange"] = bool(ok)
        res["nin"] = nin.tolist()
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_collectives_and_ghost_exchange(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        for dt in range(4):
            rc, a, b = res[r]["ar%d" % dt]
            assert rc == 0
            assert a == pytest.approx([sum(i * (k + 1) + k for k in range(world)) for i in range(5)])
            assert b == pytest.approx(list(range(5)))  # max over ranks: rank 0 holds the largest
        assert res[r]["exchange"], r
        assert min(res[r]["nin"]) > 0
