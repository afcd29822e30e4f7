"""Neutrino linear response of the force kernels (kick.f90:23-29; neutrinos/power_nu.f90
interp_tf_F :179-219 and nu_correction :449-498) against a numpy restatement, and its
effect on a kick.

Tolerances: the rescaled kernels within 2e-5 relative of interp_tf_F(|k|) * Gk computed
in float64 from the same FP32 table (the device interpolates in FP32, as the reference);
a constant transfer ratio c scales the PM velocity change by c to 2e-4 of its largest
value (the velocity changes are differences of FP32 velocities of order one); f_nu > 0 without a table scales it by 1 - f_nu (initialize.f90:316-322).
"""
import math

import numpy as np
import pytest

from cube_nu_b200.params import DEPOSIT_FIXED, config_small
from tests.helpers import lattice_state

pytestmark = pytest.mark.gpu


def _params(**kw):
    p = config_small(ng=64, nnt=2, nns=2, np_nc=2, izipx=2)
    p.deposit_mode = DEPOSIT_FIXED
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _interp_tf(klog, tlog, kr):
    """interp_tf_F: quadratic in log-log through the three table points nearest log k."""
    kn = math.log(kr)
    nb = len(klog)
    i1, i2 = 1, nb
    while i2 - i1 > 1:
        mid = (i1 + i2) // 2
        if kn > klog[mid - 1]:
            i1 = mid
        else:
            i2 = mid
    if kn - klog[i1 - 1] < klog[i2 - 1] - kn:
        i1, i2, i3 = i1 - 1, i1, i2
    else:
        i3 = i2 + 1
    if i3 > nb:
        i1, i2, i3 = i1 - 1, i2 - 1, i3 - 1
    if i1 < 1:
        i1, i2, i3 = 1, 2, 3
    K = [float(klog[i - 1]) for i in (i1, i2, i3)]
    T = [float(tlog[i - 1]) for i in (i1, i2, i3)]
    a1 = (T[0] - T[1]) / (K[0] - K[1])
    a2 = (T[1] - T[2]) / (K[1] - K[2])
    k2 = (a1 - a2) / (K[0] - K[2])
    b2 = a1 - k2 * (K[0] + K[1])
    c2 = T[0] - k2 * K[0] ** 2 - b2 * K[0]
    return math.exp(k2 * kn * kn + b2 * kn + c2)


def _table():
    kh = np.logspace(-3, 2, 300)
    tf = 0.92 + 0.08 / (1 + (kh / 0.1) ** 2)  # a smooth suppression towards 1 - f_nu at high k
    return kh, tf


@pytest.mark.parametrize("level,iapm", [(1, 2), (2, 2), (3, 2), (3, 4)])
def test_rescaled_kernels_match_restatement(level, iapm):
    from cube_nu_b200._lib import Context

    p = _params()
    st = lattice_state(p, seed=1)
    p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
    kh, tf = _table()
    with Context(p) as ctx:
        ctx.upload(*st)
        gk = ctx.green(level, iapm)
        ctx.nu_transfer(kh, tf)
        got = ctx.kernel_table(level, iapm)
    klog = np.log(kh).astype(np.float32)
    tlog = np.log(tf).astype(np.float32)
    n = gk.shape[0]
    size = {1: p.box, 2: p.box / p.nnt, 3: p.box / p.nnt / p.nns}[level]
    rng = np.random.default_rng(level * 10 + iapm)
    for _ in range(400):
        i, j, k = int(rng.integers(0, n // 2 + 1)), int(rng.integers(0, n)), int(rng.integers(0, n))
        if i == j == k == 0:
            continue
        kv = [np.float32(((m + 1 + n // 2) % n - n // 2 - 1) * (2 * math.pi / size)) for m in (i, j, k)]
        kr = float(np.sqrt(np.float32(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2])))
        want = _interp_tf(klog, tlog, kr) * float(gk[k, j, i])
        assert abs(float(got[k, j, i]) - want) <= 2e-5 * abs(want) + 1e-30, (i, j, k)
    assert got[0, 0, 0] == 1.0  # nu_correction leaves the zero mode at 1


def test_transfer_scales_the_pm_kick():
    from cube_nu_b200._lib import Context

    p = _params(pp_on=False)
    st = lattice_state(p, seed=2, disp=0.3)
    p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
    kh = np.logspace(-3, 2, 50)

    def dv(tf=None, f_nu=0.0):
        q = _params(pp_on=False, f_nu=f_nu)
        q.mass_p_cdm = p.mass_p_cdm
        with Context(q) as ctx:
            ctx.upload(*st)
            if tf is not None:
                ctx.nu_transfer(kh, np.full(kh.shape, tf))
            ctx.kick(0.2, 0.05)
            return ctx.download()[1].astype(np.float64) - st[1]

    d1 = dv()
    scale = np.abs(d1).max()
    assert np.abs(dv(tf=0.9) - 0.9 * d1).max() < 2e-4 * scale
    assert np.abs(dv(f_nu=0.05) - 0.95 * d1).max() < 2e-4 * scale
    assert np.abs(dv(tf=1.0) - d1).max() < 2e-4 * scale
