"""Zel'dovich initial conditions in CUBE's particle format (utilities/ic.f90).

Steps, as in ic.f90 for one image (nn=1):
  noise U[0,1) on the (nic*ng)^3 grid (ic.f90:262-268; here a seeded Philox stream)
  -> Box-Muller pairs along x (:289-299)
  -> forward FFT, multiply by sqrt(P(k) (nw/box)^3), zero mode (:363-385)
  -> potential kernel -4 pi / k_discrete^2 (:415-437) and inverse FFT
  -> 2x2x2 corner gradient at the particle lattice, displacement -grad/(8 nic pi ratio_cs)
     in coarse cells and velocity -grad/(8 pi nic)*vfactor(a) (:665-722)
  -> ZIPX encode floor(xq/x_resolution) with integer wrap (:717-719), PID (:723-729),
     cell order with the reference's arrival order (tile-major, spine index).
The FFTs run in numpy (small grids) or torch on a GPU (large grids); the IC is an
input to the timed step, not part of it.
"""
from __future__ import annotations

import math

import numpy as np

from . import cosmology
from .params import Params


def philox4x32_10(ctr: np.ndarray, key: tuple[int, int]):
    """Philox4x32-10 (Salmon et al. 2011) on uint64 arrays holding 32-bit lanes; ctr is
    (4, n).  The device generator (csrc/ic.cuh) computes the same function."""
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
    mask = np.uint64(0xFFFFFFFF)
    c0, c1, c2, c3 = (ctr[i].astype(np.uint64) for i in range(4))
    k0, k1 = np.uint64(key[0] & 0xFFFFFFFF), np.uint64(key[1] & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(M0) * c0
        p1 = np.uint64(M1) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & mask, lo1, (hi0 ^ c3 ^ k1) & mask, lo0
        k0 = (k0 + np.uint64(W0)) & mask
        k1 = (k1 + np.uint64(W1)) & mask
    return c0, c1, c2, c3


def noise_field(n: int, seed: int) -> np.ndarray:
    """Uniform [0,1) float32 noise on an n^3 grid, array[z, y, x] (x fastest, as
    noise_<img>.bin stores it).  Counter = Box-Muller pair index m (cells 2m, 2m+1),
    key = seed; u(2m) and u(2m+1) are the top 24 bits of the first two Philox outputs,
    the same stream the device IC (cube_gpu_ic) draws."""
    m = np.arange(n * n * n // 2, dtype=np.uint64)
    ctr = np.stack([m & np.uint64(0xFFFFFFFF), m >> np.uint64(32), np.zeros_like(m), np.zeros_like(m)])
    r0, r1, _, _ = philox4x32_10(ctr, (seed & 0xFFFFFFFF, seed >> 32))
    u = np.empty(n * n * n, dtype=np.float32)
    u[0::2] = (r0 >> np.uint64(8)).astype(np.float32) * np.float32(2.0 ** -24)
    u[1::2] = (r1 >> np.uint64(8)).astype(np.float32) * np.float32(2.0 ** -24)
    return u.reshape(n, n, n)


def pk_table(p: Params, a: float, nw: int, npts: int = 4096):
    """Linear P(k) at scale factor a on a log grid covering the IC grid's modes (the
    table format of Pcb_ic.txt: k in h/Mpc, P in (Mpc/h)^3)."""
    kmin = 2 * math.pi / p.box * 0.5
    kmax = 2 * math.pi / p.box * nw * math.sqrt(3.0)
    k = np.logspace(math.log10(kmin), math.log10(kmax), npts)
    return k, cosmology.linear_power(k, a, p)


def box_muller(u: np.ndarray) -> np.ndarray:
    """ic.f90:289-299: pairs (i, i+1) along x."""
    th = 2 * np.pi * u[..., 0::2].astype(np.float64)
    r = np.sqrt(-2 * np.log(1 - u[..., 1::2].astype(np.float64)))
    g = np.empty(u.shape, dtype=np.float32)
    g[..., 0::2] = (r * np.cos(th)).astype(np.float32)
    g[..., 1::2] = (r * np.sin(th)).astype(np.float32)
    return g


def _kgrid(n: int):
    k = np.fft.fftfreq(n, d=1.0 / n)  # integer wavenumbers, Nyquist negative
    kx = np.arange(n // 2 + 1, dtype=np.float64)
    return k, kx


def potential_field(p: Params, a: float, seed: int, use_torch: bool = False) -> np.ndarray:
    """phi on the (nic*ng)^3 IC grid, array[z, y, x] float32."""
    nw = p.nic * p.ng
    g = box_muller(noise_field(nw, seed))
    k1, kx = _kgrid(nw)
    kz = k1[:, None, None]
    ky = k1[None, :, None]
    kxx = kx[None, None, :]
    kr = 2 * math.pi * np.sqrt(kxx ** 2 + ky ** 2 + kz ** 2) / p.box
    tk, tp = pk_table(p, a, nw)
    with np.errstate(divide="ignore"):
        lp = np.interp(np.log(np.where(kr > 0, kr, tk[0])), np.log(tk), np.log(tp))  # ic.f90 interp_tf, log-log
    tf = np.sqrt(np.exp(lp) * (nw / p.box) ** 3)
    s = np.sin(np.pi * np.arange(nw) / nw)
    kdisc = (2 * s[None, None, : nw // 2 + 1]) ** 2 + (2 * np.sin(np.pi * k1 / nw))[None, :, None] ** 2 \
        + (2 * np.sin(np.pi * k1 / nw))[:, None, None] ** 2
    kdisc = np.maximum(kdisc, 1.0 / nw ** 2)
    kern = -4 * np.pi / kdisc
    kern[0, 0, 0] = 0.0
    mult = (tf * kern).astype(np.float64)
    mult[0, 0, 0] = 0.0
    if use_torch:
        import torch

        dev = torch.device("cuda")
        gt = torch.from_numpy(g).to(dev)
        ck = torch.fft.rfftn(gt.double(), dim=(0, 1, 2))
        ck *= torch.from_numpy(mult).to(dev)
        phi = torch.fft.irfftn(ck, s=(nw, nw, nw), dim=(0, 1, 2)).float().cpu().numpy()
        del gt, ck
        torch.cuda.empty_cache()
        return phi
    ck = np.fft.rfftn(g.astype(np.float64))
    ck *= mult
    return np.fft.irfftn(ck, s=(nw, nw, nw)).astype(np.float32)


def zeldovich(p: Params, z_i: float = 49.0, seed: int = 1, use_torch: bool = False):
    """Particles (xp, vp, pid, rhoc) in the reference checkpoint layout, plus header info.

    Returns a dict with keys xp (N,3) int8/int16, vp (N,3) float32, pid (N,) int64,
    rhoc (nnt^3 * nt^3,) int32, a, mass_p_cdm, vz_max, dt_vmax.
    """
    p.validate()
    a = 1.0 / (1.0 + z_i)
    nic, rcs, npnc = p.nic, p.ratio_cs, p.np_nc
    nw = nic * p.ng
    phi = potential_field(p, a, seed, use_torch)
    nlat = p.nc * npnc  # particles per dimension
    step = rcs * nic // npnc  # IC cells per lattice spacing
    idx = (np.arange(nlat) * step)  # 0-based IC index ii-1 of lattice point
    # corner gradient gradphi(d) = 0.5*sum over the 2x2x2 block of +/- phi (ic.f90:665-667)
    im = (idx - 1) % nw
    i0 = idx % nw
    P = phi  # [z,y,x]

    def blk(zs, ys, xs):
        return P[np.ix_(zs, ys, xs)].astype(np.float64)

    c = {}
    for bz, zs in ((0, im), (1, i0)):
        for by, ys in ((0, im), (1, i0)):
            for bx, xs in ((0, im), (1, i0)):
                c[(bz, by, bx)] = blk(zs, ys, xs)
    gx = sum(0.5 * (1 if bx else -1) * v for (bz, by, bx), v in c.items())
    gy = sum(0.5 * (1 if by else -1) * v for (bz, by, bx), v in c.items())
    gz = sum(0.5 * (1 if bz else -1) * v for (bz, by, bx), v in c.items())
    del c
    grad = np.stack([gx, gy, gz], axis=-1).astype(np.float32)  # [z,y,x,3] real4 gradphi
    del gx, gy, gz
    vf = cosmology.vfactor(a, p.omega_m, p.omega_l)
    # Lagrangian position in coarse units (0-based global), ic.f90:700
    lat = np.arange(nlat, dtype=np.float64) / npnc + (0.5 / nic) / rcs
    disp = -grad.astype(np.float64) / (8 * nic * math.pi * rcs)
    X = np.empty((nlat, nlat, nlat, 3), dtype=np.float64)
    X[..., 0] = lat[None, None, :] + disp[..., 0]
    X[..., 1] = lat[None, :, None] + disp[..., 1]
    X[..., 2] = lat[:, None, None] + disp[..., 2]
    vel = (-grad / np.float32(8 * math.pi * nic) * np.float32(vf)).astype(np.float32)
    # max displacement gradient for nlayer and vz_max (ic.f90:575-590)
    grad_max = np.abs(grad).max(axis=(0, 1, 2)) * 2.0
    vmax3 = grad_max / (8 * nic * math.pi) * vf
    # cells (global 0-based), wrapped
    X = X.reshape(-1, 3)
    vel = vel.reshape(-1, 3)
    cell = np.floor(X).astype(np.int64)  # g = ceiling(xq) in 1-based == floor + 1 for non-integers
    cellw = cell % p.nc
    # PID (ic.f90:723-729): lattice coords of the particle
    lz, ly, lx = np.meshgrid(np.arange(nlat), np.arange(nlat), np.arange(nlat), indexing="ij")
    lat_idx = np.stack([lx.ravel(), ly.ravel(), lz.ravel()], axis=-1)
    iq = (lat_idx * (rcs // npnc)) % p.ng
    pid = (iq[:, 0] + p.ng * iq[:, 1] + p.ng * p.ng * iq[:, 2] + 1).astype(np.int64)
    # destination tile and arrival key (ilayer, k, j, i) in the destination tile frame
    nt = p.nt
    npt = nt * npnc
    npb = npnc
    tile = cellw // nt
    # local lattice index (0-based) of the copy whose particle lands in the tile: when a
    # tile's buffer wraps onto itself (one tile) the lattice point has two copies, and the
    # one within a lattice span of the particle's local position is the landing one
    lat_loc = lat_idx - tile * npt
    xloc = np.mod(X, p.nc) - tile * nt
    lat_loc = lat_loc + nlat * np.round((xloc - (lat_loc + 0.5) / npnc) / p.nc).astype(np.int64)
    nlayer = 2 * int(math.ceil(float(np.float32(grad_max[2])) * npnc / (8 * nic * math.pi * rcs))) + 3
    kk = lat_loc[:, 2] + npb  # 0-based from 1-npb
    ilayer = kk % nlayer
    span = npt + 2 * npb
    key = ((ilayer * span + kk) * span + (lat_loc[:, 1] + npb)) * span + (lat_loc[:, 0] + npb)
    loc = cellw - tile * nt
    order_cell = ((((tile[:, 2] * p.nnt + tile[:, 1]) * p.nnt + tile[:, 0]) * nt + loc[:, 2]) * nt
                  + loc[:, 1]) * nt + loc[:, 0]
    perm = np.lexsort((key, order_cell))
    xres = 2.0 ** (-8 * p.izipx)
    frac_code = np.floor(X / xres).astype(np.int64)  # floor(xq/x_resolution) in any frame: same low bits
    mod = 1 << (8 * p.izipx)
    code = frac_code % mod
    code = np.where(code >= mod // 2, code - mod, code).astype(p.xdtype)
    rhoc = np.bincount(order_cell, minlength=p.ncells).astype(np.int32)
    return {
        "xp": np.ascontiguousarray(code[perm]),
        "vp": np.ascontiguousarray(vel[perm]),
        "pid": np.ascontiguousarray(pid[perm]),
        "rhoc": rhoc,
        "a": a,
        "mass_p_cdm": float(p.ng) ** 3 / float(nlat ** 3),
        "vz_max": float(vmax3[2]),
        "dt_vmax": float(np.float32(0.9) * 16.0 / np.float32(max(vmax3.max(), 1e-30))),
    }


def zeldovich_torch(p: Params, z_i: float = 49.0, seed: int = 1, device: str = "cuda"):
    """The same recipe as :func:`zeldovich`, computed with torch on a GPU for large
    grids (FP32 FFTs).  Noise comes from torch's seeded Philox generator, so the
    realisation differs from the numpy path.  Returns host numpy arrays."""
    import torch

    p.validate()
    a = 1.0 / (1.0 + z_i)
    nic, rcs, npnc = p.nic, p.ratio_cs, p.np_nc
    nw = nic * p.ng
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    with torch.no_grad():
        u = torch.rand((nw, nw, nw), generator=gen, device=dev, dtype=torch.float32)
        th = 2 * math.pi * u[..., 0::2]
        r = torch.sqrt(-2 * torch.log1p(-u[..., 1::2]))
        g = torch.empty_like(u)
        g[..., 0::2] = r * torch.cos(th)
        g[..., 1::2] = r * torch.sin(th)
        del u, th, r
        ck = torch.fft.rfftn(g, dim=(0, 1, 2))
        del g
        k1 = torch.fft.fftfreq(nw, d=1.0 / nw, device=dev, dtype=torch.float64)
        kx = torch.arange(nw // 2 + 1, device=dev, dtype=torch.float64)
        s1 = (2 * torch.sin(math.pi * k1 / nw)) ** 2
        sx = (2 * torch.sin(math.pi * kx / nw)) ** 2
        for iz in range(nw):  # plane by plane to bound memory
            kr = 2 * math.pi * torch.sqrt(kx[None, :] ** 2 + k1[:, None] ** 2 + k1[iz] ** 2) / p.box
            P = torch.from_numpy(cosmology.linear_power(kr.cpu().numpy(), a, p)).to(dev)
            tf = torch.sqrt(P * (nw / p.box) ** 3)
            kd = torch.clamp(sx[None, :] + s1[:, None] + s1[iz], min=1.0 / nw ** 2)
            mult = tf * (-4 * math.pi / kd)
            if iz == 0:
                mult[0, 0] = 0.0
            ck[iz] *= mult.to(torch.float32)
        phi = torch.fft.irfftn(ck, s=(nw, nw, nw), dim=(0, 1, 2))
        del ck
        nlat = p.nc * npnc
        step = rcs * nic // npnc
        idx = torch.arange(nlat, device=dev) * step
        im = (idx - 1) % nw
        i0 = idx % nw
        grad = torch.zeros((nlat, nlat, nlat, 3), device=dev, dtype=torch.float32)
        for bz, zs in ((0, im), (1, i0)):
            for by, ys in ((0, im), (1, i0)):
                for bx, xs in ((0, im), (1, i0)):
                    blk = phi.index_select(0, zs).index_select(1, ys).index_select(2, xs)
                    grad[..., 0] += 0.5 * (1 if bx else -1) * blk
                    grad[..., 1] += 0.5 * (1 if by else -1) * blk
                    grad[..., 2] += 0.5 * (1 if bz else -1) * blk
                    del blk
        del phi
        vf = cosmology.vfactor(a, p.omega_m, p.omega_l)
        grad_max = (grad.abs().amax(dim=(0, 1, 2)) * 2.0).cpu().numpy()
        vmax3 = grad_max / (8 * nic * math.pi) * vf
        lat = torch.arange(nlat, device=dev, dtype=torch.float64) / npnc + (0.5 / nic) / rcs
        X = torch.empty((nlat, nlat, nlat, 3), device=dev, dtype=torch.float64)
        X[..., 0] = lat[None, None, :]
        X[..., 1] = lat[None, :, None]
        X[..., 2] = lat[:, None, None]
        X -= grad.double() / (8 * nic * math.pi * rcs)
        vel = (-grad / (8 * math.pi * nic) * vf).reshape(-1, 3)
        del grad
        X = X.reshape(-1, 3)
        cell = torch.floor(X).long()
        cellw = cell % p.nc
        li = torch.arange(nlat, device=dev)
        lz, ly, lx = torch.meshgrid(li, li, li, indexing="ij")
        lat_idx = torch.stack([lx.reshape(-1), ly.reshape(-1), lz.reshape(-1)], dim=-1)
        del lz, ly, lx
        iq = (lat_idx * (rcs // npnc)) % p.ng
        pid = iq[:, 0] + p.ng * iq[:, 1] + p.ng * p.ng * iq[:, 2] + 1
        nt = p.nt
        npt = nt * npnc
        npb = npnc
        tile = cellw // nt
        Xw = torch.remainder(X, float(p.nc))
        lat_loc = lat_idx - tile * npt
        lat_loc = lat_loc + nlat * torch.round((Xw - tile * nt - (lat_loc + 0.5) / npnc) / p.nc).long()
        nlayer = 2 * int(math.ceil(float(grad_max[2]) * npnc / (8 * nic * math.pi * rcs))) + 3
        kk = lat_loc[:, 2] + npb
        span = npt + 2 * npb
        key = (((kk % nlayer) * span + kk) * span + (lat_loc[:, 1] + npb)) * span + (lat_loc[:, 0] + npb)
        loc = cellw - tile * nt
        order_cell = ((((tile[:, 2] * p.nnt + tile[:, 1]) * p.nnt + tile[:, 0]) * nt + loc[:, 2]) * nt
                      + loc[:, 1]) * nt + loc[:, 0]
        kmax = int(key.max().item()) + 1
        perm = torch.argsort(order_cell * kmax + key)
        xres = 2.0 ** (-8 * p.izipx)
        mod = 1 << (8 * p.izipx)
        code = torch.floor(X / xres).long() % mod
        code = torch.where(code >= mod // 2, code - mod, code)
        rhoc = torch.bincount(order_cell, minlength=p.ncells).int()
        xdt = torch.int8 if p.izipx == 1 else torch.int16
        out = {
            "xp": code[perm].to(xdt).cpu().numpy(),
            "vp": vel[perm].cpu().numpy(),
            "pid": pid[perm].cpu().numpy(),
            "rhoc": rhoc.cpu().numpy(),
            "a": a,
            "mass_p_cdm": float(p.ng) ** 3 / float(nlat ** 3),
            "vz_max": float(vmax3[2]),
            "dt_vmax": float(np.float32(0.9) * 16.0 / np.float32(max(vmax3.max(), 1e-30))),
        }
    del X, vel, cell, cellw, lat_idx, iq, pid, tile, lat_loc, kk, key, loc, order_cell, perm, code, rhoc
    torch.cuda.empty_cache()
    return out


def zeldovich_device(ctx, p: Params, z_i: float = 49.0, seed: int = 1) -> dict:
    """Generate the ICs on the GPU (cube_gpu_ic) as the context's particle state; returns
    the header values the reference's IC writes (ic.f90:575-590, 839)."""
    import ctypes

    from . import _lib

    a = 1.0 / (1.0 + z_i)
    nw = p.nic * p.ng
    k, pk = pk_table(p, a, nw)
    k = np.ascontiguousarray(k, dtype=np.float64)
    pk = np.ascontiguousarray(pk, dtype=np.float64)
    cin = _lib.ICIn(nic=p.nic, npk=k.size, seed=seed, vfactor=cosmology.vfactor(a, p.omega_m, p.omega_l),
                    reserved=0.0, pk_k=k.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                    pk_p=pk.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    out = _lib.ICOut()
    _lib._check(ctx._lib.cube_gpu_ic(ctx._h, ctypes.byref(cin), ctypes.byref(out)), "cube_gpu_ic")
    ctx.np = int(out.nplocal)
    return {"a": a, "mass_p_cdm": float(out.mass_p_cdm), "vz_max": float(out.vz_max), "dt_vmax": float(out.dt_vmax),
            "nplocal": int(out.nplocal), "grad_max": list(out.grad_max), "nlayer": int(out.nlayer)}
