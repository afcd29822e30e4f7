"""Each KDK step as one CUDA graph (cube_params.step_graph) against the eager step.

The graph holds the whole step -- scalars up, drift, PM1, PM2, classes, the PM3 class
lists built on the device, PM3, PP, the FP64 reductions and the results copied back --
with no host synchronisation inside.  With the fixed-point deposit the eager and graph
paths must give bit-identical particle states and step outputs, step after step,
including steps whose PM3 classes outgrow the captured plan (the host then redoes PM3 and
PP over exact lists) and steps that re-capture for a new plan.
"""
import numpy as np
import pytest

from cube_nu_b200.params import DEPOSIT_FIXED, DEPOSIT_FP32, config_small
from tests.helpers import clustered_state, lattice_state

pytestmark = pytest.mark.gpu


def _params(graph, fixed=True):
    p = config_small(ng=64, nnt=2, nns=2, np_nc=2, izipx=2)
    p.deposit_mode = DEPOSIT_FIXED if fixed else DEPOSIT_FP32
    p.step_graph = graph
    return p


def _run(p, st, steps):
    from cube_nu_b200._lib import Context

    outs = []
    with Context(p) as ctx:
        ctx.upload(*st)
        vz = float(np.abs(st[1][:, 2]).max())
        dt_old = 0.0
        for dt, a_mid in steps:
            so = ctx.step(dt, dt_old, a_mid, vz)
            vz = so.vz_max
            dt_old = dt
            outs.append(so)
        return ctx.download(), outs


def _same_out(a, b):
    for f in ("dt_pm1", "dt_pm2", "dt_pm3", "dt_pp", "dt_vmax", "vz_max", "f2max_pm1", "f2max_pm2", "f2max_pm3",
              "f2max_pp", "pp_pairs", "mass_pm1", "mass_pm2", "mass_pm3"):
        assert getattr(a, f) == getattr(b, f), f
    assert list(a.napm) == list(b.napm) and list(a.momentum) == list(b.momentum)


@pytest.mark.parametrize("kind", ["lattice", "clustered"])
def test_graph_step_equals_eager_step(kind):
    p = _params(False)
    n = 24000
    st = lattice_state(p, seed=3, disp=0.3, vscale=0.5) if kind == "lattice" else \
        clustered_state(p, n, seed=9, nblob=3, sigma=0.5, frac=0.6, vscale=0.5)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    steps = [(0.3, 0.05), (0.25, 0.06), (0.3, 0.07), (0.2, 0.08)]
    ref, ref_outs = _run(p, st, steps)
    q = _params(True)
    q.mass_p_cdm = p.mass_p_cdm
    got, outs = _run(q, st, steps)
    for a, b, name in zip(got, ref, ("xp", "vp", "pid", "rhoc")):
        assert np.array_equal(a, b), name
    for a, b in zip(outs, ref_outs):
        _same_out(a, b)
        assert a.tcat[6] > 0 and a.tcat[0] > 0  # stage timers recorded by the graph


def test_graph_step_redoes_pm3_when_classes_outgrow_the_plan():
    """A state whose densest subtiles jump to higher PM3 classes between captures: the
    first step is captured for the lattice's classes, the second state is clustered, so
    the captured lists overflow and the host redoes PM3 and PP exactly."""
    from cube_nu_b200._lib import Context

    p = _params(False)
    lat = lattice_state(p, seed=5, disp=0.2, vscale=0.3)
    clu = clustered_state(p, lat[0].shape[0], seed=6, nblob=2, sigma=0.3, frac=0.8, vscale=0.3)
    p.mass_p_cdm = float(p.ng) ** 3 / lat[0].shape[0]
    q = _params(True)
    q.mass_p_cdm = p.mass_p_cdm
    res = {}
    for name, par in (("eager", p), ("graph", q)):
        with Context(par) as ctx:
            ctx.upload(*lat)
            ctx.step(0.2, 0.0, 0.05, 1.0)
            ctx.upload(*clu)  # same particle count: the captured plan is reused
            so = ctx.step(0.2, 0.2, 0.06, 1.0)
            so2 = ctx.step(0.2, 0.2, 0.07, so.vz_max)
            res[name] = (ctx.download(), so, so2)
    assert max(res["graph"][1].napm[3:6]) > 0  # the clustered state reaches classes 3..5
    for a, b in zip(res["graph"][0], res["eager"][0]):
        assert np.array_equal(a, b)
    _same_out(res["graph"][1], res["eager"][1])
    _same_out(res["graph"][2], res["eager"][2])


def test_graph_step_plain_form_runs():
    """The FP32-atomics form under graph replay: same particle order and ids as eager (the
    drift is integer-exact), velocities within FP32 reordering."""
    p = _params(False, fixed=False)
    st = lattice_state(p, seed=7, disp=0.3, vscale=0.5)
    p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
    steps = [(0.3, 0.05), (0.25, 0.06)]
    ref, _ = _run(p, st, steps)
    q = _params(True, fixed=False)
    q.mass_p_cdm = p.mass_p_cdm
    got, _ = _run(q, st, steps)
    assert np.array_equal(got[2], ref[2]) and np.array_equal(got[3], ref[3])
    d = np.abs(got[1] - ref[1]).max() / np.abs(ref[1]).max()
    assert d < 1e-5, d


@pytest.mark.parametrize("graph", [False, True])
def test_drift_range_error_is_reported_and_state_stays_consistent(graph):
    """A particle whose velocity carries it beyond the ghost depth (drift.f90:64-73) makes
    the step return CUBE_E_RANGE; the particle stays in its cell, so the device state is
    still a consistent permutation (count conserved) and the context can be stepped on."""
    from cube_nu_b200._lib import Context, CubeError

    p = _params(graph)
    st = list(lattice_state(p, seed=11, disp=0.2, vscale=0.3))
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    st[1] = st[1].copy()
    st[1][123, 0] = 1e4  # dt_mid * v / ratio_cs far beyond nt + 2 ncb cells
    with Context(p) as ctx:
        ctx.upload(*st)
        with pytest.raises(CubeError, match="ghost depth"):
            ctx.step(0.2, 0.0, 0.05, 1.0)
        xp, vp, pid, rhoc = ctx.download()
        assert int(rhoc.sum()) == n and np.array_equal(np.sort(pid), np.sort(st[2]))
        vp[np.abs(vp) > 100] = 0.0
        ctx.upload(xp, vp, pid, rhoc)
        ctx.step(0.2, 0.2, 0.06, 1.0)
