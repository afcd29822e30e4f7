"""Committed golden fixtures (tests/golden/make_golden.py): the oracle must reproduce
them exactly (CPU), and the CUDA path must match them (GPU; bit-exact for the drift and
the fixed-point density, within the parity tolerances for velocities)."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import golden_params, golden_state

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(izipx):
    return dict(np.load(os.path.join(HERE, "golden_ng32_izipx%d.npz" % izipx)))


@pytest.mark.parametrize("izipx", [1, 2])
def test_inputs_reproducible(izipx):
    g = _load(izipx)
    st = golden_state(golden_params(izipx))
    for a, k in zip(st, ("xp", "vp", "pid", "rhoc")):
        assert np.array_equal(a, g[k])


@pytest.mark.parametrize("izipx", [1, 2])
def test_oracle_matches_golden(oracle_lib, izipx):
    g = _load(izipx)
    p = golden_params(izipx)
    p.mass_p_cdm = float(g["mass_p"])
    d = oracle_lib.drift(p, g["xp"], g["vp"], g["pid"], g["rhoc"], 0.4, 0.6, float(g["vz"]))
    for a, k in zip(d, ("drift_xp", "drift_vp", "drift_pid", "drift_rhoc")):
        assert np.array_equal(a, g[k]), k
    v = d[1].copy()
    out = oracle_lib.kick(p, d[0], v, d[3], 0.6, 0.05)
    assert np.array_equal(v, g["kick_vp32"])
    assert list(out.napm) == list(g["napm"])
    vfx = d[1].copy()
    oracle_lib.kick(p, d[0], vfx, d[3], 0.6, 0.05, fixed=True)
    assert np.array_equal(vfx, g["kick_vpfx"])
    assert np.array_equal(oracle_lib.green(p, 1), g["green1"])


@pytest.mark.gpu
@pytest.mark.parametrize("izipx", [1, 2])
def test_gpu_matches_golden(izipx):
    from cube_nu_b200._lib import Context
    from cube_nu_b200.params import DEPOSIT_FIXED

    g = _load(izipx)
    for fixed in (False, True):
        p = golden_params(izipx)
        p.mass_p_cdm = float(g["mass_p"])
        if fixed:
            p.deposit_mode = DEPOSIT_FIXED
        with Context(p) as ctx:
            ctx.upload(g["xp"], g["vp"], g["pid"], g["rhoc"])
            ctx.drift(0.6, 0.4, float(g["vz"]))
            xp, vp, pid, rhoc = ctx.download()
            for a, k in ((xp, "drift_xp"), (vp, "drift_vp"), (pid, "drift_pid"), (rhoc, "drift_rhoc")):
                assert np.array_equal(a, g[k]), k
            ctx.capture(1, 0, 0)
            ctx.kick(0.6, 0.05)
            dens = ctx.captured(p.nc ** 3)
            _, v, _, _ = ctx.download()
        ref = g["kick_vpfx"] if fixed else g["kick_vp32"]
        d = ref - g["drift_vp"]
        err = np.abs((v - g["drift_vp"]) - d).max() / np.abs(d).max()
        assert err < 2e-4, err
        if fixed:
            assert np.array_equal(dens, g["pm1_density_fixed"])
