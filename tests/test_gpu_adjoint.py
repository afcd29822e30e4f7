"""The hand-written adjoint of the PM step (cube_nu_b200/adjoint.py) against an FP64
autograd reference and central finite differences.

Workload (the differentiable-PM configuration): 128^3 particles in a 256 Mpc/h box, mesh
256^3 (fine cells of 1 Mpc/h), PM only, 20 KDK steps of equal code time from z=20 to
z=0, checkpoints every 5 steps; loss = mean squared difference between the final TSC
density and the final density of a second seed; gradient with respect to the 128^3 FP32
white-noise field of the first seed.

The reference is the same forward written in FP64 torch operations (TSC scatter and
gather, rfftn/irfftn with the library's Green table, the 4-point gradient by rolls), with
torch.autograd for the gradient.  Tolerances:
  * the hand-written gradient against the FP64 autograd gradient over all 128^3 modes:
    relative L2 error < 1e-3;
  * against central differences of the FP64 loss (eps = 1e-3) on 64 random modes:
    relative L2 error over those modes < 1e-3;
  * the single-step force adjoint on a small case: < 1e-4.
"""
import json
import math

import numpy as np
import pytest
import torch
import torch.utils.checkpoint

from cube_nu_b200.params import Params

pytestmark = pytest.mark.gpu

W4 = ((4.0 / 3.0 - 1.0) / 4.0, -(4.0 / 3.0) / 2.0, (4.0 / 3.0) / 2.0, (1.0 - 4.0 / 3.0) / 4.0)
OFF = (-2, -1, 1, 2)


def _params(ng=256, box=256.0):
    p = Params(ng=ng, nnt=4, nns=4, np_nc=2, izipx=1, box=box)
    p.pp_on = False
    return p


# ---------------------------------------------------------------------------------
# FP64 reference in torch
# ---------------------------------------------------------------------------------
def _tsc(x, n):
    """cells (np,3,3) and weights (np,3,3) per dimension: cells floor(x)-1..floor(x)+1."""
    fl = torch.floor(x)
    l = x - fl
    a = 1 - l
    w = torch.stack([0.5 * a * a, 0.75 - (l - 0.5) ** 2, 0.5 * l * l], dim=-1)
    cells = torch.remainder(fl.long().unsqueeze(-1) + torch.tensor([-1, 0, 1], device=x.device), n)
    return cells, w


def _flat(cells, n):
    cx, cy, cz = cells[:, 0], cells[:, 1], cells[:, 2]  # (np,3) each
    return (cz[:, None, None, :] * n + cy[:, None, :, None]) * n + cx[:, :, None, None]  # [a,b,c] -> x,y,z


def ref_density(x, n, m):
    cells, w = _tsc(x, n)
    idx = _flat(cells, n)  # (np, 3x, 3y, 3z)
    ww = w[:, 0, :, None, None] * w[:, 1, None, :, None] * w[:, 2, None, None, :]
    rho = torch.zeros(n ** 3, dtype=x.dtype, device=x.device)
    rho = rho.index_add(0, idx.reshape(-1), (m * ww).reshape(-1))
    return rho.reshape(n, n, n)


def ref_force(x, n, m, green):
    rho = ref_density(x, n, m)
    phi = torch.fft.irfftn(torch.fft.rfftn(rho) * green, s=(n, n, n))
    fm = []
    for dim in (2, 1, 0):  # x, y, z components; array is [z, y, x]
        f = 0
        for wo, o in zip(W4, OFF):
            f = f + wo * torch.roll(phi, shifts=-o, dims=dim)
        fm.append(f.reshape(-1))
    cells, w = _tsc(x, n)
    idx = _flat(cells, n).reshape(x.shape[0], -1)
    ww = (w[:, 0, :, None, None] * w[:, 1, None, :, None] * w[:, 2, None, None, :]).reshape(x.shape[0], -1)
    return torch.stack([(f[idx] * ww).sum(1) for f in fm], dim=1)


def ref_loss(w, target, p, a0, steps, d_close, green, n, m):
    from cube_nu_b200 import adjoint as A

    op = A.ic_operator(p, w.shape[0], a0, w.device, torch.float64)
    x, v = A.zeldovich(w, p, a0, op)
    for D, K in steps:
        x = torch.remainder(x + D * v, float(n))
        v = torch.utils.checkpoint.checkpoint(lambda xx, vv, K=K: vv + K * ref_force(xx, n, m, green), x, v,
                                              use_reentrant=False)
    x = torch.remainder(x + d_close * v, float(n))
    return ((ref_density(x, n, m) - target) ** 2).mean()


# ---------------------------------------------------------------------------------
def test_force_adjoint_small():
    """d(u . F)/dx from cube_dpm_force_vjp against FP64 autograd, 32^3 particles on 64^3."""
    from cube_nu_b200 import adjoint as A

    n, m = 64, 8.0
    dpm = A.DPM(n, 1.5, m)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = (torch.rand((32 ** 3, 3), generator=g, device="cuda") * n).contiguous()
    x[:4000] = torch.remainder(20.0 + 3.0 * torch.randn((4000, 3), generator=g, device="cuda"), n)  # a clump
    u = torch.randn(x.shape, generator=g, device="cuda").contiguous()
    green = torch.from_numpy(dpm.green()).double().cuda()
    f32 = dpm.force(x)
    gx = dpm.force_vjp(x, u)
    xd = x.double().requires_grad_(True)
    fd = ref_force(xd, n, m, green)
    (fd * u.double()).sum().backward()
    ferr = float((f32.double() - fd.detach()).norm() / fd.detach().norm())
    gerr = float((gx.double() - xd.grad).norm() / xd.grad.norm())
    dpm.close()
    assert ferr < 1e-5, ferr
    assert gerr < 1e-4, gerr


def test_density_adjoint_small():
    from cube_nu_b200 import adjoint as A

    n, m = 64, 8.0
    dpm = A.DPM(n, 1.5, m)
    g = torch.Generator(device="cuda").manual_seed(4)
    x = (torch.rand((20000, 3), generator=g, device="cuda") * n).contiguous()
    lam = torch.randn((n, n, n), generator=g, device="cuda")
    rho = dpm.density(x)
    gx = dpm.density_vjp(x, lam)
    xd = x.double().requires_grad_(True)
    rd = ref_density(xd, n, m)
    (rd * lam.double()).sum().backward()
    dpm.close()
    assert float((rho.double() - rd.detach()).abs().max() / rd.detach().abs().max()) < 1e-5
    assert float((gx.double() - xd.grad).norm() / xd.grad.norm()) < 1e-5


def test_adjoint_gradient_against_fp64_autograd_and_finite_differences():
    from cube_nu_b200 import adjoint as A

    p = _params()
    n, n_lat, m = 256, 128, 8.0  # mass: ng^3 / npart (ic.f90:839)
    z0, z1, S = 20.0, 0.0, 20
    a0 = 1 / (1 + z0)
    steps, d_close = A.kdk_schedule(p, z0, z1, S)
    dpm = A.DPM(n, 1.5, m)
    green = torch.from_numpy(dpm.green()).double().cuda()
    gen = torch.Generator(device="cuda").manual_seed(1)
    w = torch.randn((n_lat,) * 3, generator=gen, device="cuda")
    gen2 = torch.Generator(device="cuda").manual_seed(2)
    w2 = torch.randn((n_lat,) * 3, generator=gen2, device="cuda")
    op32 = A.ic_operator(p, n_lat, a0)
    with torch.no_grad():  # target: the final density of the second seed
        x0, v0 = A.zeldovich(w2, p, a0, op32)
        xt = A.Simulate.apply(x0.contiguous(), v0.contiguous(), dpm, steps, d_close, 5)
        target = dpm.density(xt)
    # hand-written adjoint (FP32)
    wg = w.clone().requires_grad_(True)
    loss = A.density_loss(wg, target, dpm, p, a0, steps, d_close, every=5, op=op32)
    loss.backward()
    g_adj = wg.grad.double()
    # FP64 autograd reference
    td = target.double()
    wd = w.double().requires_grad_(True)
    loss64 = ref_loss(wd, td, p, a0, steps, d_close, green, n, m)
    loss64.backward()
    g_ref = wd.grad
    err_ref = float((g_adj - g_ref).norm() / g_ref.norm())
    # central differences of the FP64 loss on 64 random modes
    rng = np.random.default_rng(7)
    modes = rng.choice(n_lat ** 3, size=64, replace=False)
    eps = 1e-3
    fd = []
    with torch.no_grad():
        for k in modes:
            wp = w.double().clone()
            wp.view(-1)[k] += eps
            lp = ref_loss(wp, td, p, a0, steps, d_close, green, n, m)
            wp.view(-1)[k] -= 2 * eps
            lm = ref_loss(wp, td, p, a0, steps, d_close, green, n, m)
            fd.append(float((lp - lm) / (2 * eps)))
    fd = np.array(fd)
    ga = g_adj.view(-1)[torch.from_numpy(modes).cuda()].cpu().numpy()
    gr = g_ref.view(-1)[torch.from_numpy(modes).cuda()].cpu().numpy()
    err_fd = float(np.linalg.norm(ga - fd) / np.linalg.norm(fd))
    err_ref_fd = float(np.linalg.norm(gr - fd) / np.linalg.norm(fd))
    dpm.close()
    print("ADJOINT " + json.dumps({"loss32": float(loss), "loss64": float(loss64), "grad_rel_l2_vs_fp64": err_ref,
                                   "fd_rel_l2": err_fd, "fp64_autograd_fd_rel_l2": err_ref_fd,
                                   "fd_max_rel": float(np.max(np.abs(ga - fd)) / np.max(np.abs(fd)))}))
    assert abs(float(loss) - float(loss64)) < 1e-4 * float(loss64)
    assert err_ref < 1e-3, err_ref
    assert err_fd < 1e-3, err_fd
