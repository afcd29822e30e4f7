"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle (oracle/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this
module.  It is the checker, never the product: the product library
(cube_nu_b200/libcube_gpu.so) does not load it.

Parity status: unpinned (no reference golden data exists; see cube_oracle.cpp).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from cube_nu_b200.params import CParams, Params

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class KickOut(ctypes.Structure):
    _fields_ = [
        ("t_pm1", ctypes.c_double), ("t_pm2", ctypes.c_double), ("t_pm3", ctypes.c_double), ("t_pp", ctypes.c_double),
        ("f2max_pm1", ctypes.c_double), ("f2max_pm2", ctypes.c_double), ("f2max_pm3", ctypes.c_double),
        ("f2max_pp", ctypes.c_double), ("vmax", ctypes.c_double * 3),
        ("dt_pm1", ctypes.c_float), ("dt_pm2", ctypes.c_float), ("dt_pm3", ctypes.c_float),
        ("dt_pp", ctypes.c_float), ("dt_vmax", ctypes.c_float), ("vz_max", ctypes.c_float),
        ("napm", ctypes.c_int32 * 8), ("pp_pairs", ctypes.c_int64), ("err", ctypes.c_int64),
        ("mass", ctypes.c_double * 3),
    ]


def build(force: bool = False) -> str:
    """(Re)build liboracle.so with its Makefile; make skips it when it is up to date."""
    path = os.path.join(_HERE, "liboracle.so")
    if force and os.path.exists(path):
        os.unlink(path)
    subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


def lib():
    global _LIB
    if _LIB is None:
        path = build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(CParams)
        vp = ctypes.c_void_p
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_green.argtypes = [P, ctypes.c_int, ctypes.c_int, vp]
        L.oracle_rfft3.argtypes = [ctypes.c_int, vp, vp]
        L.oracle_irfft3.argtypes = [ctypes.c_int, vp, vp]
        L.oracle_drift.restype = ctypes.c_int64
        L.oracle_drift.argtypes = [P, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   vp, vp, vp, vp]
        L.oracle_drift_sample.restype = ctypes.c_int64
        L.oracle_drift_sample.argtypes = [P, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                          vp, vp, vp, vp, ctypes.c_int64]
        L.oracle_drift64.restype = ctypes.c_int64
        L.oracle_drift64.argtypes = L.oracle_drift.argtypes
        L.oracle_kick.argtypes = [P, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.POINTER(KickOut), ctypes.c_int, ctypes.c_int64,
                                  ctypes.c_int, vp, ctypes.c_int64]
        L.oracle_kick64.argtypes = [P, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                    ctypes.POINTER(KickOut), ctypes.c_int, ctypes.c_int64, ctypes.c_int, vp,
                                    ctypes.c_int64]
        L.oracle_classify.argtypes = [P, vp, vp, vp]
        L.oracle_zipv_encode.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_float]
        L.oracle_zipv_decode.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_float]
        L.oracle_power.restype = ctypes.c_int64
        L.oracle_power.argtypes = [P, vp, vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, vp, vp, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]
        _LIB = L
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(n)


def green(p: Params, level: int, iapm: int = 2) -> np.ndarray:
    n = {1: p.nc, 2: p.ngt}.get(level) or p.nft(iapm)
    out = np.zeros((n, n, n // 2 + 1), dtype=np.float32)
    cp = p.to_c()
    rc = lib().oracle_green(ctypes.byref(cp), level, iapm, _ptr(out))
    if rc:
        raise RuntimeError("oracle_green failed %d" % rc)
    return out


def rfft3(r: np.ndarray) -> np.ndarray:
    n = r.shape[0]
    r = np.ascontiguousarray(r, dtype=np.float64)
    c = np.zeros((n, n, n // 2 + 1), dtype=np.complex128)
    lib().oracle_rfft3(n, _ptr(r), _ptr(c))
    return c


def irfft3(c: np.ndarray) -> np.ndarray:
    n = c.shape[0]
    c = np.ascontiguousarray(c, dtype=np.complex128).copy()
    r = np.zeros((n, n, n), dtype=np.float64)
    lib().oracle_irfft3(n, _ptr(c), _ptr(r))
    return r


def drift(p: Params, xp, vp, pid, rhoc, dt_old: float, dt: float, vz_max: float):
    """drift.f90; returns (xp, vp, pid, rhoc) in the new order."""
    n = xp.shape[0]
    fp64 = vp.dtype == np.float64
    xo = np.zeros_like(xp)
    vo = np.zeros_like(vp)
    po = np.zeros_like(pid)
    ro = np.zeros_like(rhoc)
    cp = p.to_c()
    fn = lib().oracle_drift64 if fp64 else lib().oracle_drift
    m = fn(ctypes.byref(cp), _ptr(np.ascontiguousarray(xp)), _ptr(np.ascontiguousarray(vp)),
           _ptr(np.ascontiguousarray(pid)), _ptr(np.ascontiguousarray(rhoc)), dt_old, dt, vz_max,
           _ptr(xo), _ptr(vo), _ptr(po), _ptr(ro))
    if m < 0:
        raise RuntimeError("oracle drift failed: %d" % m)
    if m != n:
        raise RuntimeError("particle count not conserved: %d -> %d" % (n, m))
    return xo, vo, po, ro


def drift_sample(p: Params, xp, vp, pid, rhoc, dt_old: float, dt: float, vz_max: float, tiles: int) -> int:
    """drift.f90 over the first `tiles` tiles only (CPU-baseline sample); returns the
    number of particles placed."""
    xo = np.zeros_like(xp)
    vo = np.zeros_like(vp)
    po = np.zeros_like(pid)
    ro = np.zeros_like(rhoc)
    cp = p.to_c()
    m = lib().oracle_drift_sample(ctypes.byref(cp), _ptr(np.ascontiguousarray(xp)), _ptr(np.ascontiguousarray(vp)),
                                  _ptr(np.ascontiguousarray(pid)), _ptr(np.ascontiguousarray(rhoc)), dt_old, dt,
                                  vz_max, _ptr(xo), _ptr(vo), _ptr(po), _ptr(ro), tiles)
    if m < 0:
        raise RuntimeError("oracle drift failed: %d" % m)
    return int(m)


def kick(p: Params, xp, vp, rhoc, dt: float, a_mid: float, fixed: bool = False, only: int = 15,
         boxes_frac: float = 0.0, debug=None):
    """kick.f90 in FP32 (vp float32, updated in place) or FP64 (vp float64).

    debug=(level, box, what, n) returns the requested field as the 2nd value."""
    out = KickOut()
    cp = p.to_c()
    dbg = np.zeros(debug[3], dtype=np.float32) if debug else None
    dl, db, dw, dn = (debug[0], debug[1], debug[2], debug[3]) if debug else (0, -1, -1, 0)
    xp = np.ascontiguousarray(xp)
    rhoc = np.ascontiguousarray(rhoc)
    if vp.dtype == np.float64:
        rc = lib().oracle_kick64(ctypes.byref(cp), _ptr(xp), _ptr(vp), _ptr(rhoc), dt, a_mid, only,
                                 ctypes.byref(out), dl, db, dw, _ptr(dbg) if dbg is not None else None, dn)
    else:
        rc = lib().oracle_kick(ctypes.byref(cp), _ptr(xp), _ptr(vp), _ptr(rhoc), dt, a_mid, int(fixed), only,
                               boxes_frac, ctypes.byref(out), dl, db, dw,
                               _ptr(dbg) if dbg is not None else None, dn)
    if rc:
        raise RuntimeError("oracle kick failed: %d (err bits %d)" % (rc, out.err))
    return (out, dbg) if debug else out


def classify(p: Params, rhoc):
    ires = np.zeros(p.ns3, dtype=np.int32)
    napm = np.zeros(8, dtype=np.int32)
    cp = p.to_c()
    lib().oracle_classify(ctypes.byref(cp), _ptr(np.ascontiguousarray(rhoc)), _ptr(ires), _ptr(napm))
    return ires, napm


def zipv_encode(v, sigma_vi: float):
    v = np.ascontiguousarray(v, dtype=np.float32)
    out = np.empty(v.shape, dtype=np.int16)
    lib().oracle_zipv_encode(_ptr(v), _ptr(out), v.size, sigma_vi)
    return out


def zipv_decode(code, sigma_vi: float):
    code = np.ascontiguousarray(code, dtype=np.int16)
    out = np.empty(code.shape, dtype=np.float32)
    lib().oracle_zipv_decode(_ptr(code), _ptr(out), code.size, sigma_vi)
    return out


class PowerOut:
    """xi is xi(10,0:nbin) as rows per bin (shape (nbin+1, 10)); see oracle/power.cpp."""

    def __init__(self, xi, delta, mean, alpha, n_done):
        self.xi, self.delta, self.mean, self.alpha, self.n_done = xi, delta, mean, alpha, n_done


def power(p: Params, xp, rhoc, nw: int, n_interp: int = 2, n_int: int = 3, n_corr: int = 4, fixed: bool = False,
          want_delta: bool = False) -> PowerOut:
    """CIC power spectrum of the particles (cicpower.f90 + powerspectrum.f90 auto_power)."""
    xp = np.ascontiguousarray(xp)
    rhoc = np.ascontiguousarray(rhoc, dtype=np.int32)
    nbin = int(round(float(np.float32(nw // 2) * np.sqrt(np.float32(3)))))
    xi = np.zeros((nbin + 2, 10), dtype=np.float32)
    delta = np.empty(nw ** 3, dtype=np.float32) if want_delta else None
    mean, alpha, done = ctypes.c_double(), ctypes.c_float(), ctypes.c_int()
    cp = p.to_c()
    nb = lib().oracle_power(ctypes.byref(cp), _ptr(xp), _ptr(rhoc), int(xp.shape[0]), nw, n_interp, n_int, n_corr,
                            int(fixed), _ptr(xi), _ptr(delta) if delta is not None else None, ctypes.byref(mean),
                            ctypes.byref(alpha), ctypes.byref(done))
    if nb < 0:
        raise ValueError("bad power-spectrum arguments")
    return PowerOut(xi[:nb + 1].copy(), delta.reshape(nw, nw, nw) if delta is not None else None, mean.value,
                    alpha.value, done.value)


def int2real(p: Params, xp, rhoc) -> np.ndarray:
    """utilities/int2real.f90:68-86: xv = real(4)((int(xp+ishift)+rshift)*x_resolution + cell),
    coarse-cell units, particles in storage order (tile z,y,x, then cell z,y,x)."""
    xp = np.asarray(xp)
    u = xp.astype(np.int64) & (0xFF if p.izipx == 1 else 0xFFFF)
    frac = (u.astype(np.float64) + 0.5) * 2.0 ** (-8 * p.izipx)
    nt, nnt = p.nt, p.nnt
    s = np.arange(p.nc ** 3, dtype=np.int64)
    i, j, k = s % nt, (s // nt) % nt, (s // nt ** 2) % nt
    t = s // nt ** 3
    tx, ty, tz = t % nnt, (t // nnt) % nnt, t // nnt ** 2
    cell = np.stack([tx * nt + i, ty * nt + j, tz * nt + k], axis=-1)
    counts = np.asarray(rhoc, dtype=np.int64).ravel()
    g = np.repeat(cell, counts, axis=0)
    return (frac + g).astype(np.float32)
