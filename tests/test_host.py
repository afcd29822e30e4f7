"""Host-side pieces: Philox known answers, expansion table and timestep, checkpoint
round trip, P(k) table."""
import os

import numpy as np

from cube_nu_b200 import checkpoint, cosmology, ic
from cube_nu_b200.params import Params


def test_philox_known_answers():
    """Random123's published Philox4x32-10 test vectors."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in kat:
        c = np.array(ctr, dtype=np.uint64).reshape(4, 1)
        got = tuple(int(x[0]) for x in ic.philox4x32_10(c, key))
        assert got == want


def test_noise_is_uniform():
    u = ic.noise_field(32, seed=5)
    assert u.dtype == np.float32 and u.min() >= 0 and u.max() < 1
    assert abs(u.mean() - 0.5) < 0.01 and abs(u.var() - 1 / 12) < 0.005


def test_timestep_reaches_checkpoint():
    tab = cosmology.expansion_table(0.6817, 0.3013, 5.0467e-5)
    bg = cosmology.Background.from_table(tab)
    st = cosmology.StepState(a=1 / 50.0)
    bg.init_cursor(st.a)
    n = 0
    while not st.final_step and n < 200:
        cosmology.timestep(bg, st, [49.0, 10.0])
        n += 1
        assert st.dt > 0
        assert st.a_mid > 0
    assert st.final_step and abs(1 / st.a - 1 - 10.0) < 1e-3
    # expansion-limited: da/a <= ra_max per step (timestep.f90:21-33)
    assert n >= 10


def test_checkpoint_round_trip(tmp_path):
    p = Params(ng=32, nnt=1, nns=2, np_nc=2, izipx=2)
    from tests.helpers import uniform_state

    xp, vp, pid, rhoc = uniform_state(p, 500, seed=1)
    h = checkpoint.new_header(nplocal=500, npglobal=500, izipx=2, izipv=2, a=0.02, mass_p_cdm=8.0)
    ck = checkpoint.Checkpoint(h, xp, vp, rhoc, pid)
    checkpoint.write(str(tmp_path), 1, 49.0, ck)
    assert os.path.getsize(checkpoint.output_name(str(tmp_path), 1, 49.0, "info")) == 224
    back = checkpoint.read(str(tmp_path), 1, 49.0, 2)
    assert np.array_equal(back.xp, xp) and np.array_equal(back.vp, vp)
    assert np.array_equal(back.pid, pid) and np.array_equal(back.rhoc, rhoc)
    try:
        checkpoint.read(str(tmp_path), 1, 49.0, 1)
        assert False, "izipx mismatch must be rejected (particle_initialization.f90:38-42)"
    except ValueError:
        pass


def test_linear_power_shape():
    p = Params()
    k = np.logspace(-3, 1, 200)
    P = cosmology.linear_power(k, 1.0, p)
    assert np.all(P > 0)
    kpk = k[np.argmax(P)]
    assert 0.01 < kpk < 0.03  # turnover near k_eq
    # growth scales as D^2
    assert np.allclose(cosmology.linear_power(k, 0.5, p) / P, (cosmology.growth_cpt(0.5, p.omega_m, p.omega_l)
                                                               / cosmology.growth_cpt(1.0, p.omega_m, p.omega_l)) ** 2)


def _bg_at(a):
    tab = cosmology.expansion_table(0.6817, 0.3013, 5.0467e-5)
    bg = cosmology.Background.from_table(tab)
    bg.init_cursor(a)
    return bg


def test_timestep_takes_the_smallest_criterion():
    """timestep.f90:34: dt = min(dt_e, dt_pm1, dt_pm2, dt_pm3, dt_refine*dt_pp, dt_vmax); each
    criterion in turn is made the smallest and must be the step taken, with dt_old the
    previous dt, the step counter advanced and a_mid = a + da/2 (timestep.f90:14-15,65)."""
    names = ("dt_pm1", "dt_pm2", "dt_pm3", "dt_pp", "dt_vmax")
    for k, name in enumerate(names):
        a0 = 1 / 40.0
        bg = _bg_at(a0)
        st = cosmology.StepState(a=a0, dt=0.0123)
        for m, other in enumerate(names):
            setattr(st, other, 0.5 + 0.1 * m)
        setattr(st, name, 1.5e-3 * (k + 1))
        cosmology.timestep(bg, st, [49.0, 0.0])
        assert st.dt == np.float32(1.5e-3 * (k + 1)), name
        assert st.dt_old == 0.0123 and st.timestep == 1
        da = st.a - a0
        assert da > 0 and abs(st.a_mid - (a0 + da / 2)) < 1e-7
        assert not st.checkpoint_step


def test_timestep_expansion_limit_matches_matter_era():
    """With every force criterion loose the step is the expansion limit ra = da/(a+da) <=
    ra_max = 0.1 (timestep.f90:20-33), below dt_max = 1.  In the code's time unit
    da/dt = (2/3) a^1.5 in the matter era (the table's omHsq*H(a)*a^3 with
    H = H0 sqrt(om) a^-1.5), so a^-1/2 falls by dt/3: ra = 0.1 (a1 = 10a/9) needs
    dt = 3 a^-1/2 (1 - sqrt(9/10)).  At a = 0.1 that is 0.487; Lambda and radiation move it
    by ~0.1%.  At a = 1/50 the same formula gives 1.09 > dt_max, so dt = dt_max there."""
    for a0, want in ((0.1, 3 / np.sqrt(0.1) * (1 - np.sqrt(0.9))), (1 / 50.0, 1.0)):
        bg = _bg_at(a0)
        st = cosmology.StepState(a=a0)
        cosmology.timestep(bg, st, [49.0, 0.0])
        da = st.a - a0
        ra = da / (a0 + da)
        assert ra <= 0.1 + 1e-6
        assert abs(st.dt - want) / want < 0.01, (a0, st.dt, want)
        if want < 1.0:
            assert ra > 0.099


def test_timestep_snaps_to_the_checkpoint():
    """A step that would pass the next checkpoint is shrunk until |(a+da)/a_next - 1| < 1e-6
    (timestep.f90:47-61); reaching the last checkpoint sets final_step."""
    a_next = 1 / 11.0
    a0 = a_next * 0.999
    bg = _bg_at(a0)
    st = cosmology.StepState(a=a0, cur_checkpoint=2)
    st.dt_pm1 = st.dt_pm2 = st.dt_pm3 = st.dt_pp = st.dt_vmax = 0.05
    cosmology.timestep(bg, st, [49.0, 10.0])
    assert st.checkpoint_step and st.final_step
    assert abs(st.a / a_next - 1) < 2e-6
    assert st.dt < 0.05
    # one checkpoint still ahead: the snap happens but the run is not over
    bg = _bg_at(a0)
    st = cosmology.StepState(a=a0, cur_checkpoint=2)
    st.dt_pm1 = st.dt_pm2 = st.dt_pm3 = st.dt_pp = st.dt_vmax = 0.05
    cosmology.timestep(bg, st, [49.0, 10.0, 5.0])
    assert st.checkpoint_step and not st.final_step


def test_expansion_table_matches_the_reference_recursion():
    """The rows t and a of the expansion table against the reference's own recursion
    (neutrinos/Pk.py:263-277, executed by tests/golden/make_expansion_golden.py with the same
    analytic H(a) standing in for CAMB): bit for bit, sampled entries and the SHA-256 of all."""
    import hashlib
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "expansion_table_ref.npz"))
    p = Params()
    tab = cosmology.expansion_table(float(g["h0"]), float(g["omega_m"]), float(g["omega_r"]))
    n = int(g["n"])
    a = np.ascontiguousarray(tab[1][:n])
    assert a[n - 1] <= 1.0 / 301 < a[n - 2]  # the table stops where Pk.py's loop does
    idx = g["idx"]
    assert np.array_equal(a[idx], g["a_sample"])
    assert np.array_equal(tab[0][idx], g["t_sample"])
    assert hashlib.sha256(a.tobytes()).hexdigest() == str(g["a_sha256"])
    assert p.h0 == float(g["h0"]) and p.omega_m == float(g["omega_m"])
