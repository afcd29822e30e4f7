"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

Tolerances:
  * drift (cell sort, arrival order, ZIPX update): bit-exact.
  * fixed-point deposit (chosen form): bit-exact density.
  * FP32 deposit: per-cell relative 1e-5 (atomics change the summation order).
  * potential: max |diff| <= 2e-5 * max |phi| (FP32 FFT rounding vs the oracle's FFT).
  * velocities after a kick: max |dv_gpu - dv_oracle| <= 2e-4 * max |dv_oracle|.
"""
import numpy as np
import pytest

from cube_nu_b200.params import DEPOSIT_FIXED, DEPOSIT_FP32, config_small
from tests.helpers import clustered_state, lattice_state, state_from_positions, uniform_state

pytestmark = pytest.mark.gpu


def _params(izipx=1, fixed=False, n=None, **kw):
    p = config_small(ng=64, nnt=2, nns=2, np_nc=2, izipx=izipx)
    for k, v in kw.items():
        setattr(p, k, v)
    p.deposit_mode = DEPOSIT_FIXED if fixed else DEPOSIT_FP32
    p.mass_p_cdm = float(p.ng) ** 3 / float(n if n else p.npglobal)
    return p


def _ctx(p, st):
    from cube_nu_b200._lib import Context

    ctx = Context(p)
    ctx.upload(*st)
    return ctx


@pytest.mark.parametrize("level,iapm", [(1, 2), (2, 2), (3, 2), (3, 3), (3, 4), (3, 5)])
def test_green_tables(oracle_lib, level, iapm):
    p = _params()
    st = lattice_state(p, seed=1)
    with _ctx(p, st) as ctx:
        g = ctx.green(level, iapm)
    ref = oracle_lib.green(p, level, iapm)
    assert g.shape == ref.shape
    scale = np.abs(ref).max()
    assert np.abs(g - ref).max() <= 1e-6 * scale
    assert g.flat[0] == 0.0


@pytest.mark.parametrize("izipx", [1, 2])
@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_drift_bitexact(oracle_lib, izipx, kind):
    p = _params(izipx=izipx)
    n = 20000
    st = uniform_state(p, n, seed=3, vscale=2.0) if kind == "uniform" else clustered_state(p, n, seed=4, vscale=2.0)
    p.mass_p_cdm = float(p.ng) ** 3 / n
    vz = float(np.abs(st[1][:, 2]).max())
    with _ctx(p, st) as ctx:
        cur = st
        for step, (dt_old, dt) in enumerate([(0.0, 1.0), (1.0, 0.7), (0.7, 1.3)]):
            ref = oracle_lib.drift(p, *cur, dt_old, dt, vz)
            ctx.drift(dt, dt_old, vz)
            got = ctx.download()
            for a, b, name in zip(got, ref, ("xp", "vp", "pid", "rhoc")):
                assert np.array_equal(a, b), "step %d: %s differs at %d entries" % (step, name, int((a != b).sum()))
            cur = ref


@pytest.mark.parametrize("max_segment", [0, 40])
def test_drift_long_segments(oracle_lib, max_segment):
    """Destination cells of every sorter class: 2..16 arrivals (half-warp sort), 17..32
    (whole-warp sort), more than 32 (block sorter) and, with max_segment = 40, more than
    max_segment (the rank sort that dense halo cores take beyond 16384)."""
    p = _params(max_segment=max_segment)
    n = 30000
    st = clustered_state(p, n, seed=5, nblob=2, sigma=0.3, frac=0.8, vscale=1.0)
    assert st[3].max() > 32
    p.mass_p_cdm = float(p.ng) ** 3 / n
    vz = float(np.abs(st[1][:, 2]).max())
    ref = oracle_lib.drift(p, *st, 0.5, 0.5, vz)
    cnt = ref[3]
    for lo, hi in ((2, 16), (17, 32), (33, 1 << 30)):
        assert np.any((cnt >= lo) & (cnt <= hi)), (lo, hi)
    with _ctx(p, st) as ctx:
        ctx.drift(0.5, 0.5, vz)
        got = ctx.download()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def _field_cases(p):
    return [(1, 0, p.nc ** 3), (2, 0, p.ngt ** 3), (2, 7, p.ngt ** 3), (3, 0, None), (3, 37, None)]


@pytest.mark.parametrize("fixed", [False, True])
def test_density_and_potential(oracle_lib, fixed):
    p = _params(fixed=fixed)
    n = 24000
    st = clustered_state(p, n, seed=7)
    p.mass_p_cdm = float(p.ng) ** 3 / n
    ires, _ = oracle_lib.classify(p, st[3])
    for level, box, size in _field_cases(p):
        if size is None:
            size = p.nft(int(ires[box])) ** 3
        for what in (0, 1):
            _, ref = oracle_lib.kick(p, st[0], st[1].copy(), st[3], 0.1, 0.05, fixed=fixed,
                                     debug=(level, box, what, size))
            with _ctx(p, st) as ctx:
                ctx.capture(level, box, what)
                ctx.kick(0.1, 0.05)
                got = ctx.captured(size)
            assert got.size == size
            if what == 0:
                if fixed:
                    assert np.array_equal(got, ref), "fixed-point density differs (level %d box %d)" % (level, box)
                else:
                    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())
                assert abs(got.sum() - ref.sum()) <= 1e-5 * abs(ref.sum()) + 1e-3
            else:
                err = np.abs(got - ref).max() / np.abs(ref).max()
                assert err < 2e-5, "phi rel err %.3g (level %d box %d)" % (err, level, box)


def test_pm3_density_dense_blob(oracle_lib):
    """A blob of 20000 particles (sigma 0.3 coarse cells) puts one subtile in a heavy class
    (rsf 6, where gridsize is inexact and the deposit takes the FP64 path for every test)
    and gives its regions more candidate particles than the 32-bit split sums allow (the
    64-bit shared-memory sums); the fixed-point density of that box and of a neighbour that
    holds the blob's ghost particles is bit-exact."""
    p = _params(fixed=True)
    rng = np.random.default_rng(21)
    c = np.array([5.4, 9.6, 2.5])  # inside subtile (1, 0, 0) of tile (0, 1, 0)
    X = np.concatenate([c + rng.normal(size=(20000, 3)) * 0.3, rng.random((6000, 3)) * p.nc])
    st = state_from_positions(p, X, rng.normal(size=X.shape))
    p.mass_p_cdm = float(p.ng) ** 3 / X.shape[0]
    ires, _ = oracle_lib.classify(p, st[3])

    def sub_of(g):
        t, l = g // p.nt, g % p.nt
        u = l // (p.nt // p.nns)
        T = (t[2] * p.nnt + t[1]) * p.nnt + t[0]
        return int(((T * p.nns + u[2]) * p.nns + u[1]) * p.nns + u[0])

    box = sub_of(np.floor(c).astype(int))
    nb = sub_of(np.floor(c).astype(int) + np.array([-2, 0, 0]))
    assert ires[box] >= 4, ires[box]
    for b in (box, nb):
        size = p.nft(int(ires[b])) ** 3
        _, ref = oracle_lib.kick(p, st[0], st[1].copy(), st[3], 0.1, 0.05, fixed=True, debug=(3, b, 0, size))
        with _ctx(p, st) as ctx:
            ctx.capture(3, b, 0)
            ctx.kick(0.1, 0.05)
            got = ctx.captured(size)
        assert np.array_equal(got, ref), "fixed-point density differs (box %d class %d)" % (b, int(ires[b]))


@pytest.mark.parametrize("izipx,fixed,kind", [(1, False, "lattice"), (2, True, "lattice"), (1, False, "clustered"),
                                              (2, True, "clustered")])
def test_kick_matches_oracle(oracle_lib, izipx, fixed, kind):
    p = _params(izipx=izipx, fixed=fixed)
    if kind == "lattice":
        st = lattice_state(p, seed=11, disp=0.3)
    else:
        st = clustered_state(p, 30000, seed=12, sigma=0.4)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    dt, a_mid = 0.2, 0.05
    v_ref = st[1].copy()
    out = oracle_lib.kick(p, st[0], v_ref, st[3], dt, a_mid, fixed=fixed)
    v64 = st[1].astype(np.float64)
    oracle_lib.kick(p, st[0], v64, st[3], dt, a_mid)
    with _ctx(p, st) as ctx:
        so = ctx.kick(dt, a_mid)
        _, v_gpu, _, _ = ctx.download()
    dref = v_ref - st[1]
    scale = np.abs(dref).max()
    err = np.abs((v_gpu - st[1]) - dref).max() / scale
    assert err < 2e-4, "kick rel err vs FP32 oracle %.3g" % err
    err64 = np.abs((v_gpu - st[1]) - (v64 - st[1])).max() / scale
    assert err64 < 2e-4, "kick rel err vs FP64 oracle %.3g" % err64
    assert list(so.napm) == list(out.napm)
    for a, b in ((so.f2max_pm1, out.f2max_pm1), (so.f2max_pm2, out.f2max_pm2), (so.f2max_pm3, out.f2max_pm3)):
        assert abs(a - b) <= 1e-4 * abs(b)
    assert abs(so.f2max_pp - out.f2max_pp) <= 1e-3 * abs(out.f2max_pp) + 1e-12
    # the oracle counts a pair once per subtile that evaluates it (kick.f90:516-566), the
    # GPU once per physical particle: out <= gpu <= 2*out
    assert out.pp_pairs <= so.pp_pairs <= 2 * out.pp_pairs


def test_step_sequence(oracle_lib):
    """Three drift+kick steps; positions agree exactly except where a rounded
    displacement flips because the FP32 kicks differ in their last bits."""
    p = _params(izipx=2)
    st = lattice_state(p, seed=21, disp=0.3, vscale=0.5)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    cur = st
    vz = float(np.abs(st[1][:, 2]).max())
    dt_old = 0.0
    with _ctx(p, st) as ctx:
        for k in range(3):
            dt, a_mid = 0.3, 0.05 + 0.01 * k
            cur = oracle_lib.drift(p, *cur, dt_old, dt, vz)
            vref = cur[1].copy()
            out = oracle_lib.kick(p, cur[0], vref, cur[3], dt, a_mid)
            cur = (cur[0], vref, cur[2], cur[3])
            so = ctx.step(dt, dt_old, a_mid, vz)
            vz = out.vz_max
            dt_old = dt
        xg, vg, pg, rg = ctx.download()
    same = np.mean(np.all(xg == cur[0], axis=1))
    assert same > 0.999
    assert np.array_equal(rg, cur[3]) or np.abs(rg - cur[3]).sum() <= 0.002 * n
    assert abs(so.vz_max - out.vz_max) <= 1e-4 * out.vz_max


def _all_class_state(p, seed=31):
    """Uniform background plus three dense clumps sized to put subtiles in PM3 classes
    3, 4 and 5 (max coarse-cell count >= 24*64, 114*64, 320*64; kick.f90:116-130)."""
    rng = np.random.default_rng(seed)
    parts = [rng.random((12000, 3)) * p.nc]
    for count, centre in ((2000, (2.5, 2.5, 2.5)), (8000, (10.5, 2.5, 10.5)), (21000, (2.5, 10.5, 10.5))):
        parts.append(np.asarray(centre) + (rng.random((count, 3)) - 0.5) * 0.9)
    X = np.concatenate(parts)
    V = rng.normal(size=X.shape) * 0.5
    from tests.helpers import state_from_positions

    return state_from_positions(p, X, V)


@pytest.mark.parametrize("fixed,generic", [(False, False), (True, False), (False, True)])
def test_every_pm3_class(oracle_lib, fixed, generic, monkeypatch):
    """Potential and velocities for subtiles of every class (mesh sides 48, 96, 144, 192),
    through the size-specialised FFT passes and, with CUBE_FFT_GENERIC=1, the generic
    Stockham passes."""
    if generic:
        monkeypatch.setenv("CUBE_FFT_GENERIC", "1")
    p = _params(fixed=fixed)
    st = _all_class_state(p)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    ires, napm = oracle_lib.classify(p, st[3])
    assert all(napm[c] > 0 for c in (2, 3, 4, 5)), list(napm)
    for cls in (2, 3, 4, 5):
        box = int(np.nonzero(ires == cls)[0][0])
        size = p.nft(cls) ** 3
        _, ref = oracle_lib.kick(p, st[0], st[1].copy(), st[3], 0.1, 0.05, fixed=fixed, debug=(3, box, 1, size))
        with _ctx(p, st) as ctx:
            ctx.capture(3, box, 1)
            ctx.kick(0.1, 0.05)
            got = ctx.captured(size)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 2e-5, "class %d phi rel err %.3g" % (cls, err)
    v_ref = st[1].copy()
    oracle_lib.kick(p, st[0], v_ref, st[3], 0.1, 0.05, fixed=fixed)
    with _ctx(p, st) as ctx:
        ctx.kick(0.1, 0.05)
        _, v_gpu, _, _ = ctx.download()
    d = v_ref - st[1]
    err = np.abs((v_gpu - st[1]) - d).max() / np.abs(d).max()
    assert err < 2e-4, err


@pytest.mark.parametrize("geom", ["proxy", "ng1024"])
def test_potential_at_bench_sizes(oracle_lib, geom):
    """FFT sizes of the 512^3 benchmark: PM2 tiles of 288^3 and PM3 subtiles of 144^3
    (one-tile geometry), and the PM1 mesh of 256^3 (ng=1024)."""
    from cube_nu_b200.params import Params
    from tests.helpers import uniform_state

    if geom == "proxy":
        p = Params(ng=256, nnt=1, nns=4, np_nc=2, izipx=2, box=250.0)
        cases = [(1, 0, p.nc ** 3, 1), (2, 0, p.ngt ** 3, 3), (3, 5, p.nft(2) ** 3, 7)]
    else:
        p = Params(ng=1024, nnt=4, nns=4, np_nc=2, izipx=2, box=1000.0)
        cases = [(1, 0, p.nc ** 3, 1)]
    n = 40000
    st = uniform_state(p, n, seed=41)
    p.mass_p_cdm = float(p.ng) ** 3 / (p.nc * p.np_nc) ** 3
    for level, box, size, only in cases:
        _, ref = oracle_lib.kick(p, st[0], st[1].copy(), st[3], 0.1, 0.05, only=only, debug=(level, box, 1, size))
        with _ctx(p, st) as ctx:
            ctx.capture(level, box, 1)
            ctx.kick(0.1, 0.05)
            got = ctx.captured(size)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 2e-5, "%s level %d phi rel err %.3g" % (geom, level, err)


def test_zipv_codec_matches_oracle(oracle_lib):
    p = _params()
    st = lattice_state(p, seed=3)
    rng = np.random.default_rng(9)
    v = (rng.normal(size=300000) * 3.0).astype(np.float32)
    sigma = 0.41
    with _ctx(p, st) as ctx:
        code = ctx.zipv_encode(v, sigma)
        back = ctx.zipv_decode(code, sigma)
        xp, code_ck, pid, rhoc = ctx.download_zipv(sigma)
    ref_code = oracle_lib.zipv_encode(v, sigma)
    # FP64 atan/tan differ from the host's libm by at most an ulp: codes agree except
    # where the unrounded value sits on a half-integer
    assert np.mean(code == ref_code) > 0.9999 and np.abs(code.astype(int) - ref_code).max() <= 1
    ref_back = oracle_lib.zipv_decode(code, sigma)
    assert np.abs(back - ref_back).max() <= 1e-6 * np.abs(ref_back).max()
    assert np.array_equal(pid, st[2]) and np.array_equal(rhoc, st[3])
    ck_ref = oracle_lib.zipv_encode(st[1], sigma)
    assert np.abs(code_ck.astype(int) - ck_ref).max() <= 1


@pytest.mark.parametrize("izipx", [1, 2])
def test_device_ic_matches_host_ic(izipx):
    """cube_gpu_ic against the numpy IC (same Philox noise and P(k) table; FP32 vs FP64
    FFT): same particles (PIDs), codes within one step, velocities to 1e-4."""
    from cube_nu_b200 import ic
    from cube_nu_b200._lib import Context
    from cube_nu_b200.params import Params

    p = Params(ng=64, nnt=2, nns=2, np_nc=2, izipx=izipx, box=100.0, nic=2)
    host = ic.zeldovich(p, z_i=49.0, seed=11)
    p.mass_p_cdm = host["mass_p_cdm"]
    with Context(p) as ctx:
        dev = ic.zeldovich_device(ctx, p, z_i=49.0, seed=11)
        xp, vp, pid, rhoc = ctx.download()
    assert dev["nplocal"] == host["xp"].shape[0]
    assert abs(dev["mass_p_cdm"] - host["mass_p_cdm"]) < 1e-6
    assert np.array_equal(np.sort(pid), np.sort(host["pid"]))
    oh, od = np.argsort(host["pid"]), np.argsort(pid)
    dx = np.abs(xp[od].astype(np.int64) - host["xp"][oh].astype(np.int64))
    mod = 1 << (8 * izipx)
    dx = np.minimum(dx, mod - dx)
    assert dx.max() <= (1 if izipx == 1 else 8)
    assert np.mean(dx == 0) > (0.999 if izipx == 1 else 0.5)
    dv = np.abs(vp[od] - host["vp"][oh]).max() / np.abs(host["vp"]).max()
    assert dv < 1e-4, dv
    # same cell occupancy except particles on a cell face
    assert np.abs(rhoc - host["rhoc"]).sum() <= 0.001 * pid.size
    assert abs(dev["vz_max"] - host["vz_max"]) <= 1e-3 * host["vz_max"]


@pytest.mark.parametrize("izipx", [1, 2])
def test_int2real_matches_oracle(oracle_lib, izipx):
    """utilities/int2real.f90:68-86 on the resident particles, after a drift reorders
    them: bit-identical to the restatement on the downloaded state."""
    p = _params(izipx=izipx)
    st = clustered_state(p, 20000, seed=61)
    with _ctx(p, st) as ctx:
        ctx.drift(0.3, 0.5, float(np.abs(st[1][:, 2]).max()))
        xv = ctx.int2real()
        xp, _, _, rhoc = ctx.download()
    ref = oracle_lib.int2real(p, xp, rhoc)
    assert xv.shape == ref.shape and xv.dtype == np.float32
    assert np.array_equal(xv, ref)
    assert xv.min() >= 0.0 and xv.max() < p.nc


@pytest.mark.parametrize("fixed", [False, True])
def test_fp64_mass_and_momentum(oracle_lib, fixed):
    """FP64 global reductions of the step: the density summed over each level's physical
    cells (particle_mesh.f90:106, kick.f90:687-688) equals the oracle's, exactly with the
    fixed-point deposit (int64 sums) and to 1e-6 relative in FP32 (the oracle, as the
    reference, sums cells that were accumulated in FP32, ~5e-8 relative off; the GPU sums
    the FP32 weights in FP64); it is the particle count up to the rounding of the TSC
    weights.  Momentum is the FP64 sum of vp after the kick."""
    p = _params(fixed=fixed)
    n = 24000
    st = clustered_state(p, n, seed=17)
    p.mass_p_cdm = float(p.ng) ** 3 / n
    ref = oracle_lib.kick(p, st[0], st[1].copy(), st[3], 0.1, 0.05, fixed=fixed)
    with _ctx(p, st) as ctx:
        so = ctx.kick(0.1, 0.05)
        _, vp, _, _ = ctx.download()
        so2 = ctx.kick(0.1, 0.05)
    got = (so.mass_pm1, so.mass_pm2, so.mass_pm3)
    for lvl in range(3):
        assert abs(got[lvl] - n) < 1e-6 * n, (lvl, got[lvl])
        if fixed:
            assert got[lvl] == ref.mass[lvl], (lvl, got[lvl], ref.mass[lvl])
        else:
            assert abs(got[lvl] - ref.mass[lvl]) < 1e-6 * n, (lvl, got[lvl], ref.mass[lvl])
    mom = vp.astype(np.float64).sum(axis=0)
    scale = np.abs(vp).astype(np.float64).sum(axis=0)
    for d in range(3):
        assert abs(so.momentum[d] - mom[d]) <= 1e-12 * scale[d], (d, so.momentum[d], mom[d])
    # deterministic: the same density gives the same sums on a second kick
    if fixed:
        assert (so2.mass_pm1, so2.mass_pm2, so2.mass_pm3) == got
