"""CUBE checkpoint files for one image (checkpoint.f90:11-39, particle_initialization.f90:31-90).

Per image the reference writes stream-unformatted files
``<opath>/image<i>/<z %7.3f>_<name>_<i>.bin`` (basic_functions.f08:97-135):
  info : the ``sim_header`` record, 16 x int64 then 24 x real32 = 224 bytes
         (parameters.f90:183-210)
  xp   : int(izipx)(3, nplocal)
  vp   : real32(3, nplocal)
  np   : int32 rhoc(nt,nt,nt,nnt,nnt,nnt) (physical cells only)
  id   : int64 pid(nplocal)
This module reads and writes them byte for byte.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

HEADER_DTYPE = np.dtype([
    ("nplocal", "<i8"), ("npglobal", "<i8"), ("izipx", "<i8"), ("izipv", "<i8"), ("image", "<i8"),
    ("nn", "<i8"), ("nnt", "<i8"), ("nt", "<i8"), ("ncell", "<i8"), ("ncb", "<i8"), ("timestep", "<i8"),
    ("cur_checkpoint", "<i8"), ("cur_halofind", "<i8"), ("cur_powerpoint", "<i8"), ("calculate_PK", "<i8"),
    ("cic_iapm", "<i8"),
    ("a", "<f4"), ("t", "<f4"), ("tau", "<f4"), ("dt_pp", "<f4"), ("dt_pm3", "<f4"), ("dt_pm2", "<f4"),
    ("dt_pm1", "<f4"), ("dt_vmax", "<f4"), ("mass_p_cdm", "<f4"), ("m_nu", "<f4", (3,)), ("Mass_nu", "<f4"),
    ("box", "<f4"), ("h0", "<f4"), ("omega_m", "<f4"), ("omega_nu", "<f4"), ("omega_l", "<f4"), ("s8", "<f4"),
    ("vsim2phys", "<f4"), ("sigma_vres", "<f4"), ("sigma_vi", "<f4"), ("z_i", "<f4"), ("vz_max", "<f4"),
])
assert HEADER_DTYPE.itemsize == 224


def z2str(z: float) -> str:
    """basic_functions.f08:49-55: write(str,'(f7.3)') z, trimmed."""
    return ("%7.3f" % z).strip()


def output_name(opath: str, image: int, z: float, name: str) -> str:
    return os.path.join(opath, "image%d" % image, "%s_%s_%d.bin" % (z2str(z), name, image))


@dataclasses.dataclass
class Checkpoint:
    header: np.ndarray  # structured scalar of HEADER_DTYPE
    xp: np.ndarray      # (N,3) int8/int16
    vp: np.ndarray      # (N,3) float32
    rhoc: np.ndarray    # (nc^3,) int32 in reference order
    pid: np.ndarray     # (N,) int64


def new_header(**kw) -> np.ndarray:
    h = np.zeros((), dtype=HEADER_DTYPE)
    for k, v in kw.items():
        h[k] = v
    return h


def write(opath: str, image: int, z: float, ck: Checkpoint) -> None:
    os.makedirs(os.path.join(opath, "image%d" % image), exist_ok=True)
    n = int(ck.header["nplocal"])
    if ck.xp.shape[0] != n or ck.vp.shape[0] != n or ck.pid.shape[0] != n:
        raise ValueError("particle arrays disagree with nplocal")
    with open(output_name(opath, image, z, "info"), "wb") as f:
        f.write(ck.header.tobytes())
    with open(output_name(opath, image, z, "xp"), "wb") as f:
        f.write(np.ascontiguousarray(ck.xp).tobytes())
    with open(output_name(opath, image, z, "vp"), "wb") as f:
        f.write(np.ascontiguousarray(ck.vp, dtype=np.float32).tobytes())
    with open(output_name(opath, image, z, "np"), "wb") as f:
        f.write(np.ascontiguousarray(ck.rhoc, dtype=np.int32).tobytes())
    with open(output_name(opath, image, z, "id"), "wb") as f:
        f.write(np.ascontiguousarray(ck.pid, dtype=np.int64).tobytes())


def read(opath: str, image: int, z: float, izipx: int) -> Checkpoint:
    """particle_initialization.f90:31-90, including the zip-format check (:38-42)."""
    with open(output_name(opath, image, z, "info"), "rb") as f:
        header = np.frombuffer(f.read(224), dtype=HEADER_DTYPE)[0].copy()
    if int(header["izipx"]) != izipx:
        raise ValueError("zip format incompatible: checkpoint izipx=%d, run izipx=%d"
                         % (int(header["izipx"]), izipx))
    n = int(header["nplocal"])
    xdt = np.int8 if izipx == 1 else np.int16
    xp = np.fromfile(output_name(opath, image, z, "xp"), dtype=xdt, count=3 * n).reshape(n, 3)
    vp = np.fromfile(output_name(opath, image, z, "vp"), dtype=np.float32, count=3 * n).reshape(n, 3)
    rhoc = np.fromfile(output_name(opath, image, z, "np"), dtype=np.int32)
    pid = np.fromfile(output_name(opath, image, z, "id"), dtype=np.int64, count=n)
    if int(rhoc.astype(np.int64).sum()) != n:
        raise ValueError("rhoc sum %d disagrees with nplocal %d" % (int(rhoc.sum()), n))
    return Checkpoint(header, xp, vp, rhoc, pid)
