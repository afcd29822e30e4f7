"""ctypes binding of the C ABI in include/cube_gpu.h (libcube_gpu.so, built in-tree).

There is no CPU fallback: if the library is missing, importing the GPU context
raises.  Build it with ``python -m cube_nu_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import CParams, Params

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcube_gpu.so")

EXPORTS = (
    "cube_params_default", "cube_gpu_create", "cube_gpu_destroy", "cube_gpu_upload", "cube_gpu_download",
    "cube_gpu_drift", "cube_gpu_kick", "cube_gpu_step", "cube_gpu_capture", "cube_gpu_captured",
    "cube_gpu_green_table", "cube_gpu_subtile_class", "cube_gpu_last_error", "cube_gpu_version",
    "cube_gpu_profile", "cube_gpu_profile_read", "cube_gpu_profile_name", "cube_gpu_kernel_launches",
    "cube_gpu_zipv_encode", "cube_gpu_zipv_decode", "cube_gpu_download_zipv", "cube_gpu_ic", "cube_gpu_power",
    "cube_gpu_int2real", "cube_gpu_step_host", "cube_gpu_pp_shape", "cube_gpu_pp_shape_get",
    "cube_gpu_nu_transfer", "cube_gpu_kernel_table", "cube_gpu_checkpoint_async", "cube_gpu_checkpoint_wait",
    "cube_gpu_set_comm", "cube_slab_cells", "cube_gpu_nplocal",
)

# cube_comm (include/cube_gpu.h): the collectives of a run split into z-slabs
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                ctypes.c_int32, ctypes.c_int32)
SENDRECV_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                               ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                               ctypes.c_int32)


class CComm(ctypes.Structure):
    _fields_ = [("user", ctypes.c_void_p), ("allreduce", ALLREDUCE_FN), ("sendrecv", SENDRECV_FN)]


class CkptFiles(ctypes.Structure):
    _fields_ = [("info", ctypes.c_char_p), ("xp", ctypes.c_char_p), ("vp", ctypes.c_char_p), ("np", ctypes.c_char_p),
                ("id", ctypes.c_char_p)]


class StepIn(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("dt_old", ctypes.c_float), ("a_mid", ctypes.c_float),
                ("vz_max", ctypes.c_float)]


class ICIn(ctypes.Structure):
    _fields_ = [("nic", ctypes.c_int32), ("npk", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("vfactor", ctypes.c_float), ("reserved", ctypes.c_float),
                ("pk_k", ctypes.POINTER(ctypes.c_double)), ("pk_p", ctypes.POINTER(ctypes.c_double))]


class ICOut(ctypes.Structure):
    _fields_ = [("nplocal", ctypes.c_int64), ("grad_max", ctypes.c_float * 3), ("vmax", ctypes.c_float * 3),
                ("vz_max", ctypes.c_float), ("dt_vmax", ctypes.c_float), ("nlayer", ctypes.c_int32),
                ("mass_p_cdm", ctypes.c_float)]


class PowerIn(ctypes.Structure):
    _fields_ = [("nw", ctypes.c_int32), ("n_interp", ctypes.c_int32), ("n_int", ctypes.c_int32),
                ("n_corr", ctypes.c_int32)]


class PowerOut(ctypes.Structure):
    _fields_ = [("nbin", ctypes.c_int64), ("mean", ctypes.c_double), ("alpha", ctypes.c_float),
                ("n_corr_done", ctypes.c_int32), ("delta_min", ctypes.c_float), ("delta_max", ctypes.c_float),
                ("ms", ctypes.c_float)]


class StepOut(ctypes.Structure):
    _fields_ = [
        ("dt_pm1", ctypes.c_float), ("dt_pm2", ctypes.c_float), ("dt_pm3", ctypes.c_float), ("dt_pp", ctypes.c_float),
        ("dt_vmax", ctypes.c_float), ("vmax", ctypes.c_float * 3), ("vz_max", ctypes.c_float),
        ("f2max_pm1", ctypes.c_float), ("f2max_pm2", ctypes.c_float), ("f2max_pm3", ctypes.c_float),
        ("f2max_pp", ctypes.c_float), ("napm", ctypes.c_int32 * 8), ("nplocal", ctypes.c_int64),
        ("pp_pairs", ctypes.c_int64), ("tcat", ctypes.c_float * 16),
        ("mass_pm1", ctypes.c_double), ("mass_pm2", ctypes.c_double), ("mass_pm3", ctypes.c_double),
        ("momentum", ctypes.c_double * 3), ("pp_candidates", ctypes.c_int64),
    ]


_LIB = None


def load():
    """Load libcube_gpu.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libcube_gpu.so not built (%s); run python -m cube_nu_b200.build" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    P = ctypes.POINTER(CParams)
    L.cube_params_default.argtypes = [P, ctypes.c_int64]
    L.cube_params_default.restype = None
    L.cube_gpu_create.argtypes = [P, ctypes.c_int, ctypes.POINTER(vp)]
    L.cube_gpu_destroy.argtypes = [vp]
    L.cube_gpu_upload.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int64]
    L.cube_gpu_download.argtypes = [vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int64)]
    L.cube_gpu_drift.argtypes = [vp, ctypes.POINTER(StepIn)]
    L.cube_gpu_kick.argtypes = [vp, ctypes.POINTER(StepIn), ctypes.POINTER(StepOut)]
    L.cube_gpu_step.argtypes = [vp, ctypes.POINTER(StepIn), ctypes.POINTER(StepOut)]
    L.cube_gpu_capture.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.cube_gpu_captured.argtypes = [vp, vp, ctypes.c_int64]
    L.cube_gpu_green_table.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int64]
    L.cube_gpu_subtile_class.argtypes = [vp, vp, ctypes.c_int64]
    L.cube_gpu_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.cube_gpu_version.restype = ctypes.c_char_p
    L.cube_gpu_profile.argtypes = [vp, ctypes.c_int]
    L.cube_gpu_profile_read.argtypes = [vp, vp, vp, ctypes.c_int]
    L.cube_gpu_profile_name.argtypes = [ctypes.c_int]
    L.cube_gpu_profile_name.restype = ctypes.c_char_p
    L.cube_gpu_kernel_launches.argtypes = [vp]
    L.cube_gpu_kernel_launches.restype = ctypes.c_int64
    L.cube_gpu_ic.argtypes = [vp, ctypes.POINTER(ICIn), ctypes.POINTER(ICOut)]
    L.cube_gpu_zipv_encode.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_float]
    L.cube_gpu_zipv_decode.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_float]
    L.cube_gpu_download_zipv.argtypes = [vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int64), ctypes.c_float]
    L.cube_gpu_power.argtypes = [vp, ctypes.POINTER(PowerIn), vp, ctypes.c_int64, vp, ctypes.POINTER(PowerOut)]
    L.cube_gpu_int2real.argtypes = [vp, vp, ctypes.c_int64]
    L.cube_gpu_step_host.argtypes = [vp, ctypes.POINTER(StepIn), ctypes.POINTER(StepOut), vp, vp, vp, vp,
                                     ctypes.c_int64]
    L.cube_gpu_pp_shape.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.cube_gpu_nu_transfer.argtypes = [vp, vp, vp, ctypes.c_int]
    L.cube_gpu_checkpoint_async.argtypes = [vp, ctypes.POINTER(CkptFiles), vp, ctypes.c_int64]
    L.cube_gpu_checkpoint_wait.argtypes = [vp]
    L.cube_gpu_kernel_table.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int64]
    L.cube_gpu_set_comm.argtypes = [vp, ctypes.POINTER(CComm)]
    L.cube_slab_cells.argtypes = [P, ctypes.c_int, vp, ctypes.c_int64]
    L.cube_slab_cells.restype = ctypes.c_int64
    L.cube_gpu_nplocal.argtypes = [vp]
    L.cube_gpu_nplocal.restype = ctypes.c_int64
    ip = ctypes.POINTER(ctypes.c_int)
    L.cube_gpu_pp_shape_get.argtypes = [vp, ctypes.c_int, ip, ip, ip, ctypes.POINTER(ctypes.c_double)]
    _LIB = L
    return L


class CubeError(RuntimeError):
    pass


def _check(rc: int, what: str) -> int:
    if rc < 0:
        buf = ctypes.create_string_buffer(512)
        load().cube_gpu_last_error(buf, 512)
        raise CubeError("%s failed (%d): %s" % (what, rc, buf.value.decode(errors="replace")))
    return rc


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """One image's device state; mirrors the reference's step subroutines."""

    def __init__(self, params: Params, device: int = 0):
        self.params = params
        self._cp = params.to_c()
        self._lib = load()
        h = ctypes.c_void_p()
        _check(self._lib.cube_gpu_create(ctypes.byref(self._cp), device, ctypes.byref(h)), "cube_gpu_create")
        self._h = h
        self.np = 0

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cube_gpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, xp, vp, pid, rhoc) -> None:
        p = self.params
        xp = np.ascontiguousarray(xp, dtype=p.xdtype)
        vp = np.ascontiguousarray(vp, dtype=np.float32)
        pid = np.ascontiguousarray(pid, dtype=np.int64)
        rhoc = np.ascontiguousarray(rhoc, dtype=np.int32)
        n = xp.shape[0]
        _check(self._lib.cube_gpu_upload(self._h, _ptr(xp), _ptr(vp), _ptr(pid), _ptr(rhoc), n), "cube_gpu_upload")
        self.np = n

    def nplocal(self) -> int:
        """Particles this context holds for its rank (what download returns)."""
        return int(_check(self._lib.cube_gpu_nplocal(self._h), "cube_gpu_nplocal"))

    def set_comm(self, comm) -> None:
        """The collectives of a run split into z-slabs (Params.nslab > 1): an object with
        ``as_c()`` returning a CComm (cube_nu_b200.slabs.TorchComm); it must outlive the
        context's steps."""
        self._comm = comm
        self._ccomm = comm.as_c()
        _check(self._lib.cube_gpu_set_comm(self._h, ctypes.byref(self._ccomm)), "cube_gpu_set_comm")

    def download(self):
        p = self.params
        self.np = self.nplocal()
        xp = np.empty((self.np, 3), dtype=p.xdtype)
        vp = np.empty((self.np, 3), dtype=np.float32)
        pid = np.empty(self.np, dtype=np.int64)
        rhoc = np.empty(p.ncells, dtype=np.int32)
        n = ctypes.c_int64()
        _check(self._lib.cube_gpu_download(self._h, _ptr(xp), _ptr(vp), _ptr(pid), _ptr(rhoc), ctypes.byref(n)),
               "cube_gpu_download")
        return xp, vp, pid, rhoc

    def drift(self, dt: float, dt_old: float, vz_max: float) -> None:
        si = StepIn(dt, dt_old, 0.0, vz_max)
        _check(self._lib.cube_gpu_drift(self._h, ctypes.byref(si)), "cube_gpu_drift")

    def kick(self, dt: float, a_mid: float) -> StepOut:
        si = StepIn(dt, 0.0, a_mid, 0.0)
        so = StepOut()
        _check(self._lib.cube_gpu_kick(self._h, ctypes.byref(si), ctypes.byref(so)), "cube_gpu_kick")
        return so

    def step(self, dt: float, dt_old: float, a_mid: float, vz_max: float) -> StepOut:
        si = StepIn(dt, dt_old, a_mid, vz_max)
        so = StepOut()
        _check(self._lib.cube_gpu_step(self._h, ctypes.byref(si), ctypes.byref(so)), "cube_gpu_step")
        return so

    def step_host(self, xp: np.ndarray, vp: np.ndarray, pid: np.ndarray, rhoc: np.ndarray, dt: float,
                  dt_old: float, a_mid: float, vz_max: float) -> StepOut:
        """One step on a host-resident state: the four arrays are uploaded, stepped and
        overwritten with the new state (cube_gpu_step_host)."""
        for a in (xp, vp, pid, rhoc):
            if not a.flags.c_contiguous:
                raise ValueError("step_host needs C-contiguous arrays")
        si = StepIn(dt, dt_old, a_mid, vz_max)
        so = StepOut()
        _check(self._lib.cube_gpu_step_host(self._h, ctypes.byref(si), ctypes.byref(so), _ptr(xp), _ptr(vp),
                                            _ptr(pid), _ptr(rhoc), ctypes.c_int64(xp.shape[0])), "cube_gpu_step_host")
        return so

    def capture(self, level: int, box: int, what: int) -> None:
        _check(self._lib.cube_gpu_capture(self._h, level, box, what), "cube_gpu_capture")

    def captured(self, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float32)
        m = _check(self._lib.cube_gpu_captured(self._h, _ptr(out), n), "cube_gpu_captured")
        return out[:m]

    def green(self, level: int, iapm: int = 2) -> np.ndarray:
        p = self.params
        n = {1: p.nc, 2: p.ngt}.get(level) or p.nft(iapm)
        out = np.empty((n, n, n // 2 + 1), dtype=np.float32)
        _check(self._lib.cube_gpu_green_table(self._h, level, iapm, _ptr(out), out.size), "cube_gpu_green_table")
        return out

    def profile(self, enable: bool = True) -> None:
        _check(self._lib.cube_gpu_profile(self._h, int(enable)), "cube_gpu_profile")

    def profile_read(self) -> dict:
        """{kernel class: (total ms, launches)} since profile(True)."""
        ms = np.zeros(64, dtype=np.float64)
        cnt = np.zeros(64, dtype=np.int64)
        k = _check(self._lib.cube_gpu_profile_read(self._h, _ptr(ms), _ptr(cnt), 64), "cube_gpu_profile_read")
        return {self._lib.cube_gpu_profile_name(i).decode(): (float(ms[i]), int(cnt[i])) for i in range(k)}

    def launches(self) -> int:
        return int(self._lib.cube_gpu_kernel_launches(self._h))

    def zipv_encode(self, v, sigma_vi: float) -> np.ndarray:
        v = np.ascontiguousarray(v, dtype=np.float32)
        out = np.empty(v.shape, dtype=np.int16)
        _check(self._lib.cube_gpu_zipv_encode(self._h, _ptr(v), _ptr(out), v.size, sigma_vi), "cube_gpu_zipv_encode")
        return out

    def zipv_decode(self, code, sigma_vi: float) -> np.ndarray:
        code = np.ascontiguousarray(code, dtype=np.int16)
        out = np.empty(code.shape, dtype=np.float32)
        _check(self._lib.cube_gpu_zipv_decode(self._h, _ptr(code), _ptr(out), code.size, sigma_vi),
               "cube_gpu_zipv_decode")
        return out

    def download_zipv(self, sigma_vi: float):
        p = self.params
        xp = np.empty((self.np, 3), dtype=p.xdtype)
        code = np.empty((self.np, 3), dtype=np.int16)
        pid = np.empty(self.np, dtype=np.int64)
        rhoc = np.empty(p.ncells, dtype=np.int32)
        n = ctypes.c_int64()
        _check(self._lib.cube_gpu_download_zipv(self._h, _ptr(xp), _ptr(code), _ptr(pid), _ptr(rhoc), ctypes.byref(n),
                                                sigma_vi), "cube_gpu_download_zipv")
        return xp, code, pid, rhoc

    def power(self, nw: int, n_interp: int = 2, n_int: int = 3, n_corr: int = 4, want_delta: bool = False):
        """Power spectrum of the resident particles (cicpower.f90 + powerspectrum.f90).

        Returns (xi, delta, out): xi has shape (nbin+1, 10), rows as xi(10,0:nbin) in the
        reference; delta is the (nw,nw,nw) density contrast or None; out a PowerOut."""
        nbin = int(round(float(np.float32(nw // 2) * np.sqrt(np.float32(3)))))
        xi = np.zeros((nbin + 2, 10), dtype=np.float32)
        delta = np.empty((nw, nw, nw), dtype=np.float32) if want_delta else None
        pin = PowerIn(nw, n_interp, n_int, n_corr)
        out = PowerOut()
        _check(self._lib.cube_gpu_power(self._h, ctypes.byref(pin), _ptr(xi), xi.size,
                                        _ptr(delta) if delta is not None else None, ctypes.byref(out)),
               "cube_gpu_power")
        return xi[:out.nbin + 1].copy(), delta, out

    def int2real(self) -> np.ndarray:
        """Real positions (np, 3) float32 in coarse-cell units (int2real.f90:68-86)."""
        out = np.empty((self.np, 3), dtype=np.float32)
        _check(self._lib.cube_gpu_int2real(self._h, _ptr(out), out.size), "cube_gpu_int2real")
        return out

    def pp_shape(self, cls: int, T: int, B: int = 256, J: int = 512) -> None:
        """Set the queue-PP shape of occupancy class cls (T <= 0: tune it again)."""
        _check(self._lib.cube_gpu_pp_shape(self._h, cls, T, B, J), "cube_gpu_pp_shape")

    def pp_shape_get(self, cls: int):
        """(T, B, J, tuned ms) of occupancy class cls, or None when it has none yet."""
        T, B, J, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        rc = _check(self._lib.cube_gpu_pp_shape_get(self._h, cls, ctypes.byref(T), ctypes.byref(B), ctypes.byref(J),
                                                    ctypes.byref(ms)), "cube_gpu_pp_shape_get")
        return (T.value, B.value, J.value, ms.value) if rc == 1 else None

    def checkpoint_async(self, opath: str, image: int, z: float, header) -> None:
        """Write the resident state as the checkpoint files of one image in the background
        (cube_gpu_checkpoint_async); names as checkpoint.output_name, header a sim_header."""
        import os

        from . import checkpoint

        os.makedirs(os.path.join(opath, "image%d" % image), exist_ok=True)
        names = {k: checkpoint.output_name(opath, image, z, k).encode() for k in ("info", "xp", "vp", "np", "id")}
        files = CkptFiles(names["info"], names["xp"], names["vp"], names["np"], names["id"])
        hb = np.ascontiguousarray(np.asarray(header)).tobytes()
        buf = ctypes.create_string_buffer(hb, len(hb))
        _check(self._lib.cube_gpu_checkpoint_async(self._h, ctypes.byref(files), ctypes.cast(buf, ctypes.c_void_p),
                                                   len(hb)), "cube_gpu_checkpoint_async")

    def checkpoint_wait(self) -> None:
        _check(self._lib.cube_gpu_checkpoint_wait(self._h), "cube_gpu_checkpoint_wait")

    def nu_transfer(self, kh, tf) -> None:
        """Neutrino transfer ratio tf_F(k) at kh (h/Mpc, increasing) for the next kicks
        (cube_gpu_nu_transfer); an empty table drops it."""
        kl = np.ascontiguousarray(np.log(np.asarray(kh, dtype=np.float64)), dtype=np.float32)
        tl = np.ascontiguousarray(np.log(np.asarray(tf, dtype=np.float64)), dtype=np.float32)
        _check(self._lib.cube_gpu_nu_transfer(self._h, _ptr(kl), _ptr(tl), kl.size), "cube_gpu_nu_transfer")

    def kernel_table(self, level: int, iapm: int = 2) -> np.ndarray:
        p = self.params
        n = {1: p.nc, 2: p.ngt}.get(level) or p.nft(iapm)
        out = np.empty((n, n, n // 2 + 1), dtype=np.float32)
        _check(self._lib.cube_gpu_kernel_table(self._h, level, iapm, _ptr(out), out.size), "cube_gpu_kernel_table")
        return out

    def subtile_class(self) -> np.ndarray:
        out = np.empty(self.params.ns3, dtype=np.int32)
        _check(self._lib.cube_gpu_subtile_class(self._h, _ptr(out), out.size), "cube_gpu_subtile_class")
        return out


def version() -> str:
    return load().cube_gpu_version().decode()
