"""Differentiable particle-mesh evolution with a hand-written adjoint (PyTorch binding).

The forward and adjoint kernels are the library's (include/cube_gpu.h, cube_dpm_*):
TSC mass assignment, the Green-table convolution between FFTs, the 4-point gradient and
TSC interpolation on one periodic mesh, in the KDK order of main.f90 (drift by the mean
of the last two steps, kick at a_mid; kick.f90 applies dv * a_mid * dt / (6 pi)).  Two
torch.autograd.Function classes expose them:

  Density  (x -> rho):       forward cube_dpm_density, backward cube_dpm_density_vjp;
  Simulate (x0, v0 -> x_end): S KDK steps and the closing half drift (main.f90:39-41);
           the backward is the symplectic adjoint of the KDK map, run from the last step
           to the first: for x' = x + D v, v' = v + K F(x'),
               lam_x += K (dF/dx')^T lam_v   (cube_dpm_force_vjp)
               lam_v += D lam_x
           with the states recomputed from checkpoints stored every `every` steps.

The initial conditions are a linear map of a white-noise field on the particle lattice
(Zel'dovich, as utilities/ic.f90 builds them: delta(k) = w(k) sqrt(P(k) (n/box)^3),
displacement i k delta / k^2, velocity = displacement * vfactor(a)), written with torch
operations so that autograd carries the gradient from (x0, v0) back to the noise.

Positions are real numbers in fine-cell units, not ZIPX codes: the quantised drift of the
production step has no derivative.  There is no CPU fallback; the library must be built.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib, cosmology
from .params import Params

_SIGS = False


def _bind(L):
    global _SIGS
    if _SIGS:
        return
    vp = ctypes.c_void_p
    L.cube_dpm_create.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.POINTER(vp)]
    L.cube_dpm_destroy.argtypes = [vp]
    L.cube_dpm_drift.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_float]
    L.cube_dpm_kdk.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_float, ctypes.c_float]
    L.cube_dpm_force.argtypes = [vp, vp, ctypes.c_int64, vp]
    L.cube_dpm_force_vjp.argtypes = [vp, vp, ctypes.c_int64, vp, vp]
    L.cube_dpm_density.argtypes = [vp, vp, ctypes.c_int64, vp]
    L.cube_dpm_density_vjp.argtypes = [vp, vp, ctypes.c_int64, vp, vp]
    L.cube_dpm_green.argtypes = [vp, vp, ctypes.c_int64]
    _SIGS = True


def _p(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def _check_xyz(t: torch.Tensor, name: str):
    if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous() or t.dim() != 2 or t.shape[1] != 3:
        raise ValueError("%s must be a contiguous CUDA float32 tensor of shape (np, 3)" % name)


class DPM:
    """One periodic n^3 PM mesh (fine-cell units) with particle mass `mass` and the
    Green table of Green/Green.f90 for softening `soft` fine cells."""

    def __init__(self, n: int, soft: float, mass: float, device: int = 0):
        self.n, self.soft, self.mass = int(n), float(soft), float(mass)
        self._lib = _lib.load()
        _bind(self._lib)
        h = ctypes.c_void_p()
        _lib._check(self._lib.cube_dpm_create(self.n, self.soft, self.mass, device, ctypes.byref(h)), "cube_dpm_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.cube_dpm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sync(self):
        torch.cuda.synchronize()  # torch's work on the inputs is done before the library reads them

    def density(self, x: torch.Tensor) -> torch.Tensor:
        _check_xyz(x, "x")
        rho = torch.empty((self.n,) * 3, dtype=torch.float32, device=x.device)
        self._sync()
        _lib._check(self._lib.cube_dpm_density(self._h, _p(x), x.shape[0], _p(rho)), "cube_dpm_density")
        return rho

    def density_vjp(self, x: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
        _check_xyz(x, "x")
        lam = lam.contiguous().float()
        gx = torch.zeros_like(x)
        self._sync()
        _lib._check(self._lib.cube_dpm_density_vjp(self._h, _p(x), x.shape[0], _p(lam), _p(gx)), "cube_dpm_density_vjp")
        return gx

    def drift(self, x: torch.Tensor, v: torch.Tensor, D: float) -> None:
        self._sync()
        _lib._check(self._lib.cube_dpm_drift(self._h, _p(x), _p(v), x.shape[0], D), "cube_dpm_drift")

    def kdk(self, x: torch.Tensor, v: torch.Tensor, D: float, K: float) -> None:
        self._sync()
        _lib._check(self._lib.cube_dpm_kdk(self._h, _p(x), _p(v), x.shape[0], D, K), "cube_dpm_kdk")

    def force(self, x: torch.Tensor) -> torch.Tensor:
        _check_xyz(x, "x")
        f = torch.empty_like(x)
        self._sync()
        _lib._check(self._lib.cube_dpm_force(self._h, _p(x), x.shape[0], _p(f)), "cube_dpm_force")
        return f

    def force_vjp(self, x: torch.Tensor, u: torch.Tensor) -> torch.Tensor:
        _check_xyz(x, "x")
        u = u.contiguous()
        gx = torch.zeros_like(x)
        self._sync()
        _lib._check(self._lib.cube_dpm_force_vjp(self._h, _p(x), x.shape[0], _p(u), _p(gx)), "cube_dpm_force_vjp")
        return gx

    def green(self) -> np.ndarray:
        n = self.n
        out = np.empty((n, n, n // 2 + 1), dtype=np.float32)
        _lib._check(self._lib.cube_dpm_green(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size), "cube_dpm_green")
        return out


class Density(torch.autograd.Function):
    """TSC density of the particles on the DPM mesh (n^3 floats)."""

    @staticmethod
    def forward(ctx, x, dpm: DPM):
        x = x.detach().contiguous()
        ctx.save_for_backward(x)
        ctx.dpm = dpm
        return dpm.density(x)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        return ctx.dpm.density_vjp(x, g), None


class Simulate(torch.autograd.Function):
    """S KDK steps and the closing half drift: (x0, v0) -> final positions.

    steps: [(D, K)] per step (drift, then kick by K * force); d_close: the closing drift.
    every: checkpoint interval of the backward recomputation."""

    @staticmethod
    def forward(ctx, x0, v0, dpm: DPM, steps, d_close: float, every: int):
        x = x0.detach().contiguous().clone()
        v = v0.detach().contiguous().clone()
        ckpt = []
        for s, (D, K) in enumerate(steps):
            if s % every == 0:
                ckpt.append((x.clone(), v.clone()))
            dpm.kdk(x, v, D, K)
        dpm.drift(x, v, d_close)
        ctx.dpm, ctx.steps, ctx.d_close, ctx.every = dpm, list(steps), d_close, every
        ctx.ckpt = ckpt
        return x

    @staticmethod
    def backward(ctx, gx):
        dpm, steps, every = ctx.dpm, ctx.steps, ctx.every
        lam_x = gx.detach().contiguous().clone()
        lam_v = torch.zeros_like(lam_x)
        lam_v += ctx.d_close * lam_x  # closing drift x_end = x + Dc v
        S = len(steps)
        for seg in reversed(range(len(ctx.ckpt))):
            s0, s1 = seg * every, min(S, (seg + 1) * every)
            x, v = ctx.ckpt[seg][0].clone(), ctx.ckpt[seg][1].clone()
            xs = []
            for s in range(s0, s1):  # recompute the positions each kick saw
                D, K = steps[s]
                dpm.drift(x, v, D)
                xs.append(x.clone())
                dpm.kdk(x, v, 0.0, K)
            for s in reversed(range(s0, s1)):
                D, K = steps[s]
                lam_x += dpm.force_vjp(xs[s - s0], K * lam_v)  # v' = v + K F(x')
                lam_v += D * lam_x                             # x' = x + D v
        ctx.ckpt = None
        return lam_x, lam_v, None, None, None, None


# ---------------------------------------------------------------------------------
# Initial conditions (linear in the noise) and the KDK schedule
# ---------------------------------------------------------------------------------
def ic_operator(p: Params, n_lat: int, a: float, device="cuda", dtype=torch.float32):
    """Per-mode factors of the Zel'dovich map on the n_lat^3 particle lattice: returns
    (kvec, mult) with the displacement (in fine cells) Psi_d = irfft(i k_d mult w(k))."""
    box = p.box
    f = np.fft.fftfreq(n_lat, d=1.0 / n_lat)
    fx = np.arange(n_lat // 2 + 1, dtype=np.float64)
    kz, ky, kx = np.meshgrid(f, f, fx, indexing="ij")
    kr = 2 * math.pi * np.sqrt(kx ** 2 + ky ** 2 + kz ** 2) / box  # h/Mpc
    with np.errstate(divide="ignore", invalid="ignore"):
        P = cosmology.linear_power(np.where(kr > 0, kr, 1.0), a, p)
    amp = np.where(kr > 0, np.sqrt(P * (n_lat / box) ** 3), 0.0)  # delta(k) per unit noise (ic.f90 tf)
    k_lat = [2 * math.pi * k / n_lat for k in (kx, ky, kz)]         # radians per lattice cell
    k2 = k_lat[0] ** 2 + k_lat[1] ** 2 + k_lat[2] ** 2
    fine = p.ng / n_lat
    with np.errstate(divide="ignore", invalid="ignore"):
        mult = np.where(k2 > 0, amp / np.where(k2 > 0, k2, 1.0), 0.0) * fine
    kv = [torch.tensor(k, dtype=dtype, device=device) for k in k_lat]
    return kv, torch.tensor(mult, dtype=dtype, device=device)


def zeldovich(w: torch.Tensor, p: Params, a: float, op=None):
    """(x0, v0), (np, 3) in fine cells, from the white noise w (n_lat^3, [z, y, x]); linear
    in w and differentiable by torch autograd.  Lattice points sit at cell centres."""
    n_lat = w.shape[0]
    kv, mult = op if op is not None else ic_operator(p, n_lat, a, w.device, w.dtype)
    wk = torch.fft.rfftn(w, dim=(0, 1, 2))
    fine = p.ng / n_lat
    disp = []
    for d in range(3):  # x, y, z
        disp.append(torch.fft.irfftn(1j * kv[d] * mult * wk, s=(n_lat,) * 3, dim=(0, 1, 2)))
    g = (torch.arange(n_lat, dtype=w.dtype, device=w.device) + 0.5) * fine
    Z, Y, X = torch.meshgrid(g, g, g, indexing="ij")
    q = torch.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], dim=1)
    psi = torch.stack([dd.reshape(-1) for dd in disp], dim=1)
    vf = cosmology.vfactor(a, p.omega_m, p.omega_l)
    x0 = torch.remainder(q + psi, float(p.ng))
    return x0, psi * vf


def kdk_schedule(p: Params, z_start: float, z_end: float, nsteps: int):
    """[(D, K)] per step and the closing drift, from equal code-time steps: D = (dt_old +
    dt)/2 (drift.f90:21), K = a_mid dt / (6 pi) (kick.f90 velocity update)."""
    tab = cosmology.expansion_table(p.h0, p.omega_m, p.omega_r)
    bg = cosmology.Background.from_table(tab)
    sched = cosmology.fixed_steps(bg, 1 / (1 + z_start), 1 / (1 + z_end), nsteps)
    steps = [((dt_old + dt) / 2, a_mid * dt / 6 / math.pi) for dt, dt_old, a_mid, _ in sched]
    return steps, sched[-1][0] / 2


def density_loss(w: torch.Tensor, target: torch.Tensor, dpm: DPM, p: Params, a0: float, steps, d_close,
                 every: int = 5, op=None) -> torch.Tensor:
    """Mean squared difference between the final TSC density and `target`."""
    x0, v0 = zeldovich(w, p, a0, op)
    x = Simulate.apply(x0.contiguous(), v0.contiguous(), dpm, steps, d_close, every)
    rho = Density.apply(x, dpm)
    return ((rho - target) ** 2).mean()
