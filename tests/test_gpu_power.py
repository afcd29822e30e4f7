"""Power spectrum on the GPU (cube_gpu_power) against the oracle restatement of
utilities/cicpower.f90 + utilities/powerspectrum.f90.

Tolerances:
  * mode counts per bin: exact.  Mean k per bin: relative 1e-4 (the oracle sums |k| in
    real(4), as the reference does).
  * mean density: relative 1e-12 (fixed point), 1e-6 (FP32 atomics).
  * delta_c: the fixed-point density is bit-identical, so delta differs by at most one
    float rounding of rho/mean - 1 (the means are summed in different orders):
    |d_gpu - d_oracle| <= 2e-7 * max(1, |d|).  FP32 atomics: 1e-5 * max(1, |d|).
  * raw power, power minus shot noise: 2e-4 relative, plus 1e-5 of the largest raw
    power (the oracle sums bins in real(4) as the reference does; the GPU in double).
  * aliasing-corrected power: 2e-3 relative plus 1e-4 of the largest raw power (alpha
    comes from the corrected power itself and feeds back through four passes).
"""
import numpy as np
import pytest

from cube_nu_b200.params import DEPOSIT_FIXED, DEPOSIT_FP32, config_small
from tests.helpers import clustered_state, lattice_state, uniform_state

pytestmark = pytest.mark.gpu


def _params(izipx, fixed, ng=64, nnt=2):
    p = config_small(ng=ng, nnt=nnt, nns=2, np_nc=2, izipx=izipx)
    p.deposit_mode = DEPOSIT_FIXED if fixed else DEPOSIT_FP32
    return p


def _run(p, st, nw, **kw):
    from cube_nu_b200._lib import Context

    p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
    with Context(p) as ctx:
        ctx.upload(*st)
        return ctx.power(nw, want_delta=True, **kw)


def _compare(xi, ref):
    assert xi.shape == ref.shape
    g, r = xi[1:], ref[1:]
    scale = np.abs(r[:, 2]).max()
    checks = {
        "count": (g[:, 0], r[:, 0], 0.0, 0.0),
        "k": (g[:, 1], r[:, 1], 1e-4, 0.0),
        "raw": (g[:, 2], r[:, 2], 2e-4, 1e-5 * scale),
        "minus shot": (g[:, 3], r[:, 3], 2e-4, 1e-5 * scale),
        "corrected": (g[:, 4], r[:, 4], 2e-3, 1e-4 * scale),
    }
    bad = []
    for name, (a, b, rtol, atol) in checks.items():
        err = np.abs(a - b)
        lim = rtol * np.abs(b) + atol
        if not np.all(err <= lim):
            bad.append("%s: worst %.3g over %.3g" % (name, float(np.max(err - lim)), float(lim[np.argmax(err - lim)])))
    assert not bad, "; ".join(bad)
    assert not np.any(g[:, 5:])


@pytest.mark.parametrize("izipx,fixed,nw", [(2, True, 32), (1, True, 64), (2, False, 48), (2, True, 128),
                                            (1, False, 192), (2, True, 72), (1, False, 108)])
def test_power_matches_oracle(oracle_lib, izipx, fixed, nw):
    """72 and 108 take the generic forward FFT (no size-specialised passes), the rest the
    size-specialised plane or row passes."""
    p = _params(izipx, fixed)
    st = clustered_state(p, 50000, seed=40 + nw, nblob=24, sigma=0.4, frac=0.8)
    xi, delta, out = _run(p, st, nw)
    if nw <= 48:
        assert out.n_corr_done == 4  # these meshes resolve the clustering above shot noise
    ref = oracle_lib.power(p, st[0], st[3], nw, fixed=fixed, want_delta=True)
    assert out.nbin == ref.xi.shape[0] - 1
    tol = (2e-7 if fixed else 1e-5) * np.maximum(1.0, np.abs(ref.delta))
    derr = float(np.max(np.abs(delta - ref.delta) - tol))
    info = "mean %.17g/%.17g alpha %.8g/%.8g passes %d/%d delta excess %.3g" % (
        out.mean, ref.mean, out.alpha, ref.alpha, out.n_corr_done, ref.n_done, derr)
    assert abs(out.mean - ref.mean) <= (1e-12 if fixed else 1e-6) * ref.mean, info
    assert derr <= 0, info
    # the correction runs only where the shot-noise-subtracted power at k_Nyq and k_Nyq/2
    # is positive (alpha finite); both sides must take the same branch
    assert out.n_corr_done == ref.n_done, info
    if ref.n_done:
        assert abs(out.alpha - ref.alpha) <= 1e-3 * abs(ref.alpha), info
    else:
        assert np.isnan(out.alpha), info
    _compare(xi, ref.xi)
    assert out.delta_min == delta.min() and out.delta_max == delta.max()


def test_power_without_correction_on_a_lattice(oracle_lib):
    """A sub-Poisson lattice has negative shot-noise-subtracted power at the Nyquist
    frequency: alpha is NaN and pk_correction leaves xi(5) = xi(4), as in the reference."""
    p = _params(2, True)
    st = lattice_state(p, seed=41, disp=0.05)
    xi, _, out = _run(p, st, 32)
    ref = oracle_lib.power(p, st[0], st[3], 32, fixed=True)
    assert np.isnan(out.alpha) and out.n_corr_done == 0
    assert np.array_equal(xi[1:, 4], xi[1:, 3])
    _compare(xi, ref.xi)


def test_power_invariants_at_proxy_size():
    """A 256^3 mesh over 2M particles (the single-tile geometry of the 512^3 run):
    every independent mode is binned once and the mean is np/nw^3."""
    p = config_small(ng=256, nnt=1, nns=4, np_nc=2, izipx=2)
    p.deposit_mode = DEPOSIT_FIXED
    n = 2_000_000
    st = uniform_state(p, n, seed=42, vscale=0.1)
    xi, delta, out = _run(p, st, 256, n_corr=1)
    nw = 256
    assert xi[:, 0].sum() == (nw ** 3 - 8) // 2 + 7
    assert abs(out.mean - n / nw ** 3) <= 1e-9 * n / nw ** 3
    assert abs(float(delta.astype(np.float64).mean())) < 1e-6
    # Poisson particles: raw power ~ shot noise, so power minus shot noise ~ 0 on average
    mid = slice(10, 100)
    assert abs(np.mean(xi[mid, 3]) / np.mean(xi[mid, 2])) < 0.05
