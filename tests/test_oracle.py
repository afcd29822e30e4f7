"""CPU tests of the oracle: FFT convention, Green invariants, drift invariants,
mass conservation (the reference's own runtime checks, kick.f90:42,72,242 and
drift.f90:139-147)."""
import numpy as np
import pytest

from cube_nu_b200.params import config_small
from tests.helpers import clustered_state, lattice_state, uniform_state


def _p(**kw):
    p = config_small(ng=64, nnt=2, nns=2, np_nc=2, izipx=1)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@pytest.mark.parametrize("n", [6, 12, 16, 48])
def test_fft_matches_numpy(oracle_lib, n):
    r = np.random.default_rng(n).random((n, n, n))
    c = oracle_lib.rfft3(r)
    assert np.abs(c - np.fft.rfftn(r)).max() < 1e-11 * n ** 3
    back = oracle_lib.irfft3(c) / n ** 3
    assert np.abs(back - r).max() < 1e-12


@pytest.mark.parametrize("level,iapm", [(1, 2), (2, 2), (3, 2), (3, 4)])
def test_green_invariants(oracle_lib, level, iapm):
    p = _p()
    g = oracle_lib.green(p, level, iapm)
    n = g.shape[0]
    assert g[0, 0, 0] == 0.0  # Green.f90:71
    assert g[n // 2, n // 2, n // 2] == 0.0
    # real-space symmetry of the kernel: G(kz,ky,kx) = G(-kz,ky,kx) = G(kz,-ky,kx)
    assert np.allclose(g[1:], g[1:][::-1], rtol=1e-5, atol=1e-7 * np.abs(g).max())
    assert np.allclose(g[:, 1:], g[:, 1:][:, ::-1], rtol=1e-5, atol=1e-7 * np.abs(g).max())
    # cubic symmetry: swap y,z
    assert np.allclose(g, np.swapaxes(g, 0, 1), rtol=1e-5, atol=1e-7 * np.abs(g).max())
    assert np.isfinite(g).all()


def test_drift_invariants(oracle_lib):
    p = _p()
    st = uniform_state(p, 8000, seed=1, vscale=3.0)
    xo, vo, po, ro = oracle_lib.drift(p, *st, 0.5, 1.0, float(np.abs(st[1][:, 2]).max()))
    assert ro.sum() == st[0].shape[0]
    assert np.array_equal(np.sort(po), np.sort(st[2]))  # PID permutation (drift.f90:185-193)
    assert (po > 0).all()
    # zero velocity: nothing moves, order unchanged
    st0 = (st[0], np.zeros_like(st[1]), st[2], st[3])
    xo, vo, po, ro = oracle_lib.drift(p, *st0, 0.5, 1.0, 0.0)
    assert np.array_equal(xo, st[0]) and np.array_equal(po, st[2]) and np.array_equal(ro, st[3])


def test_drift_rejects_far_moves(oracle_lib):
    p = _p()
    st = uniform_state(p, 1000, seed=2)
    st = (st[0], np.full_like(st[1], 100.0), st[2], st[3])
    with pytest.raises(RuntimeError):
        oracle_lib.drift(p, *st, 0.5, 1.0, 100.0)


@pytest.mark.parametrize("fixed", [False, True])
def test_mass_sums(oracle_lib, fixed):
    p = _p()
    st = clustered_state(p, 12000, seed=3)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    _, d1 = oracle_lib.kick(p, st[0], st[1].copy(), st[3], 0.1, 0.05, fixed=fixed, only=1,
                            debug=(1, 0, 0, p.nc ** 3))
    assert abs(d1.sum() - p.ng ** 3) < 1e-4 * p.ng ** 3
    assert (d1 >= 0).all()


def test_fp32_close_to_fp64(oracle_lib):
    p = _p()
    st = lattice_state(p, seed=4, disp=0.3)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    v32 = st[1].copy()
    v64 = st[1].astype(np.float64)
    oracle_lib.kick(p, st[0], v32, st[3], 0.2, 0.05)
    oracle_lib.kick(p, st[0], v64, st[3], 0.2, 0.05)
    d = v64 - st[1]
    assert np.abs((v32 - st[1]) - d).max() < 2e-4 * np.abs(d).max()


def test_classify(oracle_lib):
    p = _p()
    st = clustered_state(p, 20000, seed=5, nblob=1, sigma=0.2, frac=0.5)
    ires, napm = oracle_lib.classify(p, st[3])
    assert napm.sum() == p.ns3
    assert set(np.unique(ires)).issubset({2, 3, 4, 5})
    assert ires.max() >= 3  # a tight blob pushes a subtile into a heavier class


def test_zipv_codec_round_trip(oracle_lib):
    """ZIPV int16 velocity codec (utilities/pp_subtile.f90:61,125): codes cover
    [-32767, 32767], decode(encode(v)) is within half a code step, and encode is
    idempotent on decoded values."""
    rng = np.random.default_rng(7)
    sigma = 0.37
    v = np.concatenate([rng.normal(size=20000).astype(np.float32) * 2.0, np.array([0, 1e-6, -1e-6, 50, -50], np.float32)])
    code = oracle_lib.zipv_encode(v, sigma)
    assert code.dtype == np.int16 and abs(int(code.astype(np.int64).max())) <= 32767
    back = oracle_lib.zipv_decode(code, sigma)
    assert np.array_equal(oracle_lib.zipv_encode(back, sigma), code)
    # step of the code at v: dv/dcode = pi/65535 * (1 + (s v)^2)/s, s = sqrt(pi/2)/(2.5 sigma)
    s = np.sqrt(np.pi / 2) / (sigma * 2.5)
    step = np.pi / 65535 * (1 + (s * v.astype(np.float64)) ** 2) / s
    assert np.all(np.abs(back - v) <= 0.51 * step + 1e-6 * np.abs(v))
    assert code[np.argmin(np.abs(v))] == 0


@pytest.mark.parametrize("nw", [16, 32])
def test_power_spectrum_invariants(oracle_lib, nw):
    """cicpower + auto_power restatement: every independent mode lands in one bin
    ((nw^3-8)/2 + 7 of them for even nw), delta has zero mean, fixed-point and FP32
    deposits agree, and a sub-Poisson lattice leaves pk_correction off (alpha NaN)."""
    p = _p(izipx=2)
    st = clustered_state(p, 40000, seed=8, nblob=20, sigma=0.4, frac=0.8)
    n = st[0].shape[0]
    a = oracle_lib.power(p, st[0], st[3], nw, fixed=True, want_delta=True)
    b = oracle_lib.power(p, st[0], st[3], nw, fixed=False)
    assert a.xi[:, 0].sum() == (nw ** 3 - 8) // 2 + 7
    assert abs(a.mean - n / nw ** 3) < 1e-9 * n / nw ** 3
    assert abs(float(a.delta.astype(np.float64).mean())) < 1e-6
    assert a.n_done == 4 and np.isfinite(a.alpha)
    scale = np.abs(b.xi[1:, 2]).max()  # raw-power scale: bins near k_max hold far less power
    np.testing.assert_allclose(a.xi[1:, :5], b.xi[1:, :5], rtol=2e-4, atol=1e-5 * scale)
    lat = lattice_state(p, seed=9, disp=0.05)
    c = oracle_lib.power(p, lat[0], lat[3], nw)
    assert np.isnan(c.alpha) and c.n_done == 0
    assert np.array_equal(c.xi[1:, 4], c.xi[1:, 3])


def test_oracle_mass_sums_are_particle_count(oracle_lib):
    """The reference's mass check (kick.f90:42,72,242): each level's density summed over its
    physical cells is the particle count, up to the rounding of the TSC weights."""
    from cube_nu_b200.params import DEPOSIT_FIXED, config_small
    from tests.helpers import clustered_state

    p = config_small(ng=32, nnt=1, nns=2, np_nc=2, izipx=2)
    p.deposit_mode = DEPOSIT_FIXED
    n = 3000
    st = clustered_state(p, n, seed=2)
    p.mass_p_cdm = float(p.ng) ** 3 / n
    for fixed in (False, True):
        out = oracle_lib.kick(p, st[0], st[1].copy(), st[3], 0.1, 0.05, fixed=fixed)
        for m in out.mass:
            assert abs(m - n) < 1e-6 * n, (fixed, list(out.mass))
