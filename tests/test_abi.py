"""The C ABI library loads on a machine without a GPU and exports every entry point
that include/cube_gpu.h declares; calls that need a device fail cleanly."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cube_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cube_\w+)\s*\(", src)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("cube_gpu_create", "cube_gpu_upload", "cube_gpu_step", "cube_gpu_download", "cube_gpu_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from cube_nu_b200 import _lib

    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(declared_functions())


def test_params_default_matches_parameters_f90():
    from cube_nu_b200 import _lib
    from cube_nu_b200.params import CParams

    L = _lib.load()
    p = CParams()
    L.cube_params_default(ctypes.byref(p), 128)
    assert (p.ng, p.ratio_cs, p.nnt, p.nns, p.ncb, p.ngb, p.izipx) == (128, 4, 4, 4, 4, 16, 2)
    assert abs(p.app - 0.06) < 1e-7 and abs(p.apm1c - 3.5) < 1e-7


def test_create_rejects_bad_geometry():
    from cube_nu_b200 import _lib
    from cube_nu_b200.params import CParams

    L = _lib.load()
    p = CParams()
    L.cube_params_default(ctypes.byref(p), 100)  # 100/4=25 coarse cells do not split into 4 tiles
    p.mass_p_cdm = 8.0
    h = ctypes.c_void_p()
    rc = L.cube_gpu_create(ctypes.byref(p), 0, ctypes.byref(h))
    assert rc == -1  # CUBE_E_ARG, before any CUDA call
    buf = ctypes.create_string_buffer(256)
    L.cube_gpu_last_error(buf, 256)
    assert b"divide" in buf.value


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cube_nu_b200 import _lib
    from cube_nu_b200.params import Params

    p = Params(ng=64, nnt=2, nns=2, np_nc=2, izipx=1, mass_p_cdm=8.0)
    with pytest.raises(_lib.CubeError):
        _lib.Context(p)
