"""A run split into z-slabs (Params.nslab > 1) against the same run on one context.

The ranks are separate processes on the one GPU, talking over gloo through TorchComm
(cube_nu_b200/slabs.py); their kernels never wait on one another (every exchange goes
through the host between kernels).  With the fixed-point deposit the slabs' particles,
joined in slab order, must equal the one-context run bit for bit after several steps
(drift with ghost sources and dropped destinations, PM1 summed over ranks, PM2/PM3/PP on
each rank's tiles with ghost layers), and the reduced step results must agree: maxima
exactly, pair counts exactly, masses and momentum to FP64 rounding of the per-rank sums.
With FP32 deposits the PM1 sum over ranks rounds differently, so velocities agree to
FP32 tolerance."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from cube_nu_b200.params import DEPOSIT_FIXED, DEPOSIT_FP32, Params
from tests.helpers import clustered_state, lattice_state

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = {
    # name: (params kwargs, state, steps)
    "two_slabs_int8_queue": (dict(ng=64, nnt=2, nns=2, np_nc=2, izipx=1, pp_queue=True, deposit_mode=DEPOSIT_FIXED),
                             ("clustered", 30000, 7), 3),
    "four_slabs_int16": (dict(ng=128, nnt=4, nns=2, np_nc=2, izipx=2, pp_queue=False, deposit_mode=DEPOSIT_FIXED),
                         ("lattice", 0, 8), 2),
    "two_slabs_fp32": (dict(ng=64, nnt=2, nns=2, np_nc=2, izipx=1, pp_queue=True, deposit_mode=DEPOSIT_FP32),
                       ("clustered", 30000, 9), 2),
}
FIELDS = ("f2max_pm1", "f2max_pm2", "f2max_pm3", "f2max_pp", "vz_max", "pp_pairs", "pp_candidates", "mass_pm1",
          "mass_pm2", "mass_pm3", "dt_pm1", "dt_pp", "dt_vmax")


def _state(p, kind, n, seed):
    if kind == "clustered":
        return clustered_state(p, n, seed=seed, sigma=0.5, vscale=0.5)
    return lattice_state(p, seed=seed, disp=0.3, vscale=0.5)


def _run(p, part, steps, comm=None):
    from cube_nu_b200._lib import Context

    outs = []
    with Context(p) as ctx:
        if comm is not None:
            ctx.set_comm(comm)
        ctx.upload(*part)
        vz = float(np.abs(part[1][:, 2]).max()) if part[1].size else 0.0
        if comm is not None:  # the same drift layers on every rank: the global vz_max
            import torch
            import torch.distributed as dist

            t = torch.tensor([vz], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            vz = float(t[0])
        dt_old = 0.0
        for k in range(steps):
            dt, a_mid = 0.3, 0.05 + 0.01 * k
            so = ctx.step(dt, dt_old, a_mid, vz)
            outs.append({f: getattr(so, f) for f in FIELDS} | {"momentum": list(so.momentum), "nplocal": so.nplocal})
            vz = so.vz_max
            dt_old = dt
        return ctx.download(), outs


def _worker(rank, world, port, case, path):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from cube_nu_b200 import slabs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        kw, (kind, n, seed), steps = CASES[case]
        p = Params(**kw)
        st = _state(p, kind, n, seed)
        p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
        part = slabs.split_state(p, *st, world)[rank]
        q = slabs.slab_params(p, world, rank)
        comm = slabs.TorchComm()
        (xp, vp, pid, rhoc), outs = _run(q, part, steps, comm)
        np.savez(os.path.join(path, "r%d.npz" % rank), xp=xp, vp=vp, pid=pid, rhoc=rhoc,
                 outs=np.array([repr(o) for o in outs]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("case", list(CASES))
def test_slabs_equal_one_context(case, tmp_path):
    from cube_nu_b200 import slabs

    kw, (kind, n, seed), steps = CASES[case]
    p = Params(**kw)
    world = 4 if case.startswith("four") else 2
    st = _state(p, kind, n, seed)
    p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, str(tmp_path))) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(600)
    assert all(pr.exitcode == 0 for pr in procs), [pr.exitcode for pr in procs]
    parts, outs = [], []
    for r in range(world):
        z = np.load(os.path.join(str(tmp_path), "r%d.npz" % r))
        parts.append((z["xp"], z["vp"], z["pid"], z["rhoc"]))
        outs.append([eval(o) for o in z["outs"]])
    (xr, vr, pr_, rr), ref = _run(p, st, steps)
    xs, vs, ps, rs = slabs.join_states(parts)
    assert np.array_equal(rs, rr)
    assert np.array_equal(ps, pr_)
    fixed = kw["deposit_mode"] == DEPOSIT_FIXED
    if fixed:
        assert np.array_equal(xs, xr)
        assert np.array_equal(vs, vr)
    else:  # PM1 summed over ranks in another order: FP32 rounding of the kicks
        assert np.mean(np.all(xs == xr, axis=1)) > 0.999
        assert np.abs(vs - vr).max() <= 1e-4 * np.abs(vr).max()
    for k in range(steps):
        for r in range(world):
            o, e = outs[r][k], ref[k]
            assert sum(outs[q][k]["nplocal"] for q in range(world)) == e["nplocal"]
            for f in ("pp_pairs", "pp_candidates"):
                assert o[f] == e[f], (f, o[f], e[f])
            for f in ("f2max_pm1", "f2max_pm2", "f2max_pm3", "f2max_pp", "vz_max", "dt_pm1", "dt_pp", "dt_vmax"):
                if fixed:
                    assert o[f] == e[f], (f, o[f], e[f])
                else:
                    assert o[f] == pytest.approx(e[f], rel=1e-4)
            for f in ("mass_pm1", "mass_pm2", "mass_pm3"):
                assert o[f] == pytest.approx(e[f], rel=1e-12 if fixed else 1e-9)
            scale = max(1.0, float(np.abs(e["momentum"]).max()))
            assert np.allclose(o["momentum"], e["momentum"], rtol=0, atol=1e-9 * scale if fixed else 1e-3 * scale)
