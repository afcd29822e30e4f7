"""cube_gpu_pm1_density_noalloc: the PM1 density for callers that cannot allocate.

Some hosts cannot call cudaMalloc when they need a density field -- their device memory
is already held by another framework's caching pool, or they sit on a latency-bound path
where cudaMalloc/cudaFree would synchronise the whole device.  This entry point keeps all
of its scratch in one static device array, so the caller only passes inputs and outputs.

Each case calls it twice in a row (different particle sets, so the second call must not
see the first call's scratch) and compares both results with the density the existing
context path records (cube_gpu_capture level 1 + cube_gpu_kick + cube_gpu_captured):
bit-identical with the fixed-point deposit, per-cell relative 1e-5 with FP32 atomics.
This file is collected last so that a failure here stops a -x run after all other tests.
"""
import ctypes

import numpy as np
import pytest

from cube_nu_b200.params import DEPOSIT_FIXED, DEPOSIT_FP32, CParams, config_small
from tests.helpers import clustered_state, uniform_state

pytestmark = pytest.mark.gpu

CUBE_E_CAPACITY = -3
CUBE_E_COUNT = -5
MAX_CELLS = 262144
MAX_PARTICLES = 2097152


def _lib():
    from cube_nu_b200._lib import load

    L = load()
    f = L.cube_gpu_pm1_density_noalloc
    f.argtypes = [ctypes.POINTER(CParams), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return L


def _last_error(L):
    buf = ctypes.create_string_buffer(512)
    L.cube_gpu_last_error(buf, 512)
    return buf.value.decode()


def _params(fixed, ng=64, nnt=2, nns=2):
    p = config_small(ng=ng, nnt=nnt, nns=nns, np_nc=2, izipx=2)
    p.deposit_mode = DEPOSIT_FIXED if fixed else DEPOSIT_FP32
    return p


def _context_density(p, st):
    """PM1 density from the existing entry points (capture during a kick)."""
    from cube_nu_b200._lib import Context

    with Context(p) as ctx:
        ctx.upload(*st)
        ctx.capture(1, 0, 0)
        ctx.kick(0.1, 0.05)
        return ctx.captured(p.nc ** 3)


def _noalloc_density(L, p, st, np_arg=None):
    """Call the allocation-free entry point on device copies of st (the test, standing
    in for the caller, owns every buffer)."""
    import torch

    xp = torch.from_numpy(np.ascontiguousarray(st[0])).cuda()
    rhoc = torch.from_numpy(np.ascontiguousarray(st[3]).astype(np.int32)).cuda()
    rho = torch.full((p.nc ** 3,), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    cp = p.to_c()
    n = st[0].shape[0] if np_arg is None else np_arg
    rc = L.cube_gpu_pm1_density_noalloc(ctypes.byref(cp), xp.data_ptr(), rhoc.data_ptr(), n, rho.data_ptr(), None)
    return rc, rho.cpu().numpy()


def _compare(got, ref, fixed):
    assert got.shape == ref.shape
    if fixed:
        assert np.array_equal(got, ref), "fixed-point PM1 density differs from the context path"
    else:
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())


@pytest.mark.parametrize("fixed", [True, False])
def test_noalloc_density_matches_context_twice(fixed):
    L = _lib()
    p = _params(fixed)
    states = [clustered_state(p, 24000, seed=11), uniform_state(p, 9000, seed=12)]
    for st in states:
        p.mass_p_cdm = float(p.ng) ** 3 / st[0].shape[0]
        ref = _context_density(p, st)
        rc, got = _noalloc_density(L, p, st)
        assert rc == 0, _last_error(L)
        _compare(got, ref, fixed)
        assert abs(got.sum() - p.ng ** 3) < 1e-4 * p.ng ** 3


def test_noalloc_density_at_the_size_limit():
    """64^3 coarse cells, the largest mesh the static scratch holds (one tile of the
    512^3 workload's geometry), twice in a row."""
    L = _lib()
    p = _params(True, ng=256, nnt=1, nns=4)
    assert p.nc ** 3 == MAX_CELLS
    for seed, n in ((21, 300000), (22, 120000)):
        st = uniform_state(p, n, seed=seed, vscale=0.1)
        p.mass_p_cdm = float(p.ng) ** 3 / n
        ref = _context_density(p, st)
        rc, got = _noalloc_density(L, p, st)
        assert rc == 0, _last_error(L)
        _compare(got, ref, True)


def test_noalloc_density_rejects_oversize_and_bad_counts():
    L = _lib()
    # a mesh beyond the static scratch: rejected before any device work
    p = _params(True, ng=512, nnt=4)
    p.mass_p_cdm = 1.0
    cp = p.to_c()
    dummy = ctypes.c_void_p(16)
    rc = L.cube_gpu_pm1_density_noalloc(ctypes.byref(cp), dummy, dummy, 10, dummy, None)
    assert rc == CUBE_E_CAPACITY
    assert "static scratch" in _last_error(L)
    p = _params(True)
    p.mass_p_cdm = 1.0
    cp = p.to_c()
    rc = L.cube_gpu_pm1_density_noalloc(ctypes.byref(cp), dummy, dummy, MAX_PARTICLES + 1, dummy, None)
    assert rc == CUBE_E_CAPACITY
    # rhoc summing to more particles than np: cell indices past np are not written
    st = uniform_state(p, 5000, seed=13)
    p.mass_p_cdm = float(p.ng) ** 3 / 5000
    rc, _ = _noalloc_density(L, p, st, np_arg=4990)
    assert rc == CUBE_E_COUNT, _last_error(L)
    # a negative count whose total still equals np: rejected, not deposited around cell 0
    bad = list(st)
    r = bad[3].astype(np.int32).copy()
    r[np.flatnonzero(r > 0)[0]] += 3
    zero = np.flatnonzero(r == 0)[0]
    r[zero] = -3
    assert r.sum() == 5000 and r.min() < 0
    bad[3] = r
    rc, _ = _noalloc_density(L, p, bad)
    assert rc == CUBE_E_COUNT, _last_error(L)
    assert "negative" in _last_error(L)
    # and a valid call right after still matches the context path
    ref = _context_density(p, st)
    rc, got = _noalloc_density(L, p, st)
    assert rc == 0, _last_error(L)
    _compare(got, ref, True)
