"""The queue PP of the chosen form (cube_params.pp_queue) against the oracle's PP_Force
(kick.f90:376-588) and against itself under every shape.

Tolerances: velocities after a kick within 2e-4 of the largest velocity change of the FP32
and FP64 oracles (as the thread-per-particle PP); f2max_pp within 1e-3.  Shapes (light
threshold T, item size B, chunk J) only move work between the light and heavy kernels and
the queue, so the velocities must be bit-identical across shapes, in eager and graph steps.
"""
import numpy as np
import pytest

from cube_nu_b200.params import DEPOSIT_FIXED, config_small
from tests.helpers import clustered_state, lattice_state, state_from_positions

pytestmark = pytest.mark.gpu


def _params(izipx=1, graph=False):
    p = config_small(ng=64, nnt=2, nns=2, np_nc=2, izipx=izipx)
    p.deposit_mode = DEPOSIT_FIXED
    p.pp_queue = True
    p.step_graph = graph
    return p


def _blob_state(p, seed=31, nblob=8000):
    """A dense blob (cells of several hundred particles, the heavy path) over a uniform
    background (light cells)."""
    rng = np.random.default_rng(seed)
    c = np.array([5.4, 9.6, 2.5])
    X = np.concatenate([c + rng.normal(size=(nblob, 3)) * 0.35, rng.random((12000, 3)) * p.nc])
    return state_from_positions(p, X, rng.normal(size=X.shape) * 0.5)


def _kick(p, st, shape=None, dt=0.2, a_mid=0.05):
    from cube_nu_b200._lib import Context

    with Context(p) as ctx:
        if shape is not None:
            for cls in range(4):
                ctx.pp_shape(cls, *shape)
        ctx.upload(*st)
        so = ctx.kick(dt, a_mid)
        tuned = [ctx.pp_shape_get(c) for c in range(4)]
        return ctx.download()[1], so, tuned


@pytest.mark.parametrize("izipx,kind", [(1, "clustered"), (2, "blob"), (1, "lattice")])
def test_queue_pp_matches_oracle(oracle_lib, izipx, kind):
    p = _params(izipx)
    st = {"clustered": lambda: clustered_state(p, 30000, seed=12, sigma=0.4),
          "blob": lambda: _blob_state(p),
          "lattice": lambda: lattice_state(p, seed=11, disp=0.3)}[kind]()
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    dt, a_mid = 0.2, 0.05
    v_ref = st[1].copy()
    out = oracle_lib.kick(p, st[0], v_ref, st[3], dt, a_mid, fixed=True)
    v64 = st[1].astype(np.float64)
    oracle_lib.kick(p, st[0], v64, st[3], dt, a_mid)
    v_gpu, so, tuned = _kick(p, st)
    dref = v_ref - st[1]
    scale = np.abs(dref).max()
    assert np.abs((v_gpu - st[1]) - dref).max() / scale < 2e-4
    assert np.abs((v_gpu - st[1]) - (v64 - st[1])).max() / scale < 2e-4
    assert abs(so.f2max_pp - out.f2max_pp) <= 1e-3 * abs(out.f2max_pp) + 1e-12
    assert out.pp_pairs <= so.pp_pairs <= 2 * out.pp_pairs
    assert so.pp_candidates >= so.pp_pairs
    assert any(t is not None for t in tuned)  # the autotuner ran for this state's class


def test_queue_pp_is_shape_independent():
    """The blob puts cells of several hundred particles in the heavy path for small T; all
    shapes, from everything light (T=4096) to most particles heavy (T=4), give the same
    velocities bit for bit; the blob's particles have far more pairs in range than the
    deferred-pair columns hold, so their flushes in the middle of a cell are covered."""
    p = _params(2)
    st = _blob_state(p)
    p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
    assert st[3].max() > 256
    ref, so_ref, _ = _kick(p, st, shape=(4096, 256, 512))
    for shape in ((4, 128, 256), (16, 256, 1024), (64, 512, 32), (256, 128, 4096), (4, 32, 256), (16, 64, 64)):
        v, so, _ = _kick(p, st, shape=shape)
        assert np.array_equal(v, ref), shape
        assert so.pp_pairs == so_ref.pp_pairs and so.pp_candidates == so_ref.pp_candidates
        assert so.f2max_pp == so_ref.f2max_pp


def test_queue_pp_graph_equals_eager():
    from cube_nu_b200._lib import Context

    res = {}
    for graph in (False, True):
        p = _params(1, graph=graph)
        st = clustered_state(p, 30000, seed=13, sigma=0.4)
        p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
        with Context(p) as ctx:
            for cls in range(4):
                ctx.pp_shape(cls, 16, 256, 512)
            ctx.upload(*st)
            vz = float(np.abs(st[1][:, 2]).max())
            outs = []
            for dt, dt_old, a in ((0.2, 0.0, 0.05), (0.2, 0.2, 0.06), (0.15, 0.2, 0.07)):
                so = ctx.step(dt, dt_old, a, vz)
                vz = so.vz_max
                outs.append((so.pp_pairs, so.pp_candidates, so.f2max_pp))
            res[graph] = (ctx.download(), outs)
    for a, b in zip(res[True][0], res[False][0]):
        assert np.array_equal(a, b)
    assert res[True][1] == res[False][1]
