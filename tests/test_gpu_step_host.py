"""cube_gpu_step_host (one step on a host-resident state, with the copies the step does
not wait for overlapping it) against cube_gpu_upload + cube_gpu_step + cube_gpu_download
on the same state.  Fixed-point deposit, so every output is deterministic and the two
paths must agree bit for bit, over two steps in a row."""
import numpy as np
import pytest

from cube_nu_b200.params import DEPOSIT_FIXED, config_small
from tests.helpers import clustered_state

pytestmark = pytest.mark.gpu

STEPS = [(0.4, 0.3, 0.05), (0.5, 0.4, 0.06)]  # (dt, dt_old, a_mid)


def _setup():
    p = config_small(ng=64, nnt=2, nns=2, np_nc=2, izipx=2)
    p.deposit_mode = DEPOSIT_FIXED
    st = clustered_state(p, 30000, seed=31, sigma=0.4, vscale=0.5)
    p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
    return p, st


def _reference(p, st):
    from cube_nu_b200._lib import Context

    outs = []
    cur = [a.copy() for a in st]
    with Context(p) as ctx:
        for dt, dt_old, a_mid in STEPS:
            ctx.upload(*cur)
            vz = float(np.abs(cur[1][:, 2]).max())
            so = ctx.step(dt, dt_old, a_mid, vz)
            cur = list(ctx.download())
            outs.append(([a.copy() for a in cur], (so.dt_pm1, so.dt_pm2, so.dt_pm3, so.dt_pp, so.vz_max)))
    return outs


@pytest.mark.parametrize("pinned", [False, True])
def test_step_host_matches_upload_step_download(pinned):
    import torch
    from cube_nu_b200._lib import Context

    p, st = _setup()
    ref = _reference(p, st)
    if pinned:
        arrs = []
        for a in st:
            t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
            b = t.numpy()
            b[...] = a
            arrs.append((t, b))
        host = [b for _, b in arrs]
    else:
        host = [a.copy() for a in st]
    with Context(p) as ctx:
        for k, (dt, dt_old, a_mid) in enumerate(STEPS):
            vz = float(np.abs(host[1][:, 2]).max())
            so = ctx.step_host(*host, dt, dt_old, a_mid, vz)
            want, want_dt = ref[k]
            for got, exp, name in zip(host, want, ("xp", "vp", "pid", "rhoc")):
                assert np.array_equal(got, exp), "step %d: %s differs at %d entries" % (k, name, int((got != exp).sum()))
            assert (so.dt_pm1, so.dt_pm2, so.dt_pm3, so.dt_pp, so.vz_max) == want_dt


def test_step_host_rejects_bad_counts():
    from cube_nu_b200._lib import Context, CubeError

    p, st = _setup()
    xp, vp, pid, rhoc = [a.copy() for a in st]
    rhoc[0] += 1  # counts no longer sum to the particle number
    with Context(p) as ctx:
        with pytest.raises(CubeError, match="sum"):
            ctx.step_host(xp, vp, pid, rhoc, 0.4, 0.3, 0.05, 1.0)
        with pytest.raises(CubeError, match="before upload"):
            ctx.step(0.4, 0.3, 0.05, 1.0)
        ctx.upload(*st)  # a valid upload makes the context usable again
        ctx.step(0.4, 0.3, 0.05, float(np.abs(st[1][:, 2]).max()))
