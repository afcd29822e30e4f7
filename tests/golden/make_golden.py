"""Generate the small golden fixtures in tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

The reference's own golden data (test/baseline.tar.gz) is a git-LFS pointer without
payload and the reference cannot be built here, so these fixtures are outputs of the
oracle restatement (oracle/cube_oracle.cpp): they pin the oracle and the CUDA path
against regressions, not against a reference run.  Inputs are a seeded perturbed
lattice plus a clump (16^3 + 600 particles, ng=32, one tile).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cube_nu_b200.params import Params  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.helpers import state_from_positions  # noqa: E402


def golden_params(izipx: int) -> Params:
    p = Params(ng=32, nnt=1, nns=2, np_nc=2, izipx=izipx, box=50.0)
    return p


def golden_state(p: Params, seed: int = 2024):
    rng = np.random.default_rng(seed)
    m = p.nc * p.np_nc
    g = (np.arange(m) + 0.5) / p.np_nc
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    lat = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=-1) + rng.normal(size=(m ** 3, 3)) * 0.15
    clump = np.array([2.5, 5.5, 3.5]) + rng.normal(size=(600, 3)) * 0.25
    pos = np.concatenate([lat, clump])
    vel = rng.normal(size=pos.shape) * 0.8
    return state_from_positions(p, pos, vel)


def make(izipx: int) -> dict:
    p = golden_params(izipx)
    st = golden_state(p)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    vz = float(np.abs(st[1][:, 2]).max())
    d = O.drift(p, *st, 0.4, 0.6, vz)
    v32 = d[1].copy()
    out32 = O.kick(p, d[0], v32, d[3], 0.6, 0.05)
    vfx = d[1].copy()
    O.kick(p, d[0], vfx, d[3], 0.6, 0.05, fixed=True)
    v64 = d[1].astype(np.float64)
    O.kick(p, d[0], v64, d[3], 0.6, 0.05)
    _, dens_fx = O.kick(p, d[0], d[1].copy(), d[3], 0.6, 0.05, fixed=True, only=1, debug=(1, 0, 0, p.nc ** 3))
    return dict(
        xp=st[0], vp=st[1], pid=st[2], rhoc=st[3], mass_p=np.float32(p.mass_p_cdm), vz=np.float32(vz),
        drift_xp=d[0], drift_vp=d[1], drift_pid=d[2], drift_rhoc=d[3],
        kick_vp32=v32, kick_vpfx=vfx, kick_vp64=v64, pm1_density_fixed=dens_fx,
        green1=O.green(p, 1), napm=np.array(list(out32.napm), dtype=np.int32),
        f2max=np.array([out32.f2max_pm1, out32.f2max_pm2, out32.f2max_pm3, out32.f2max_pp]),
    )


if __name__ == "__main__":
    for izipx in (1, 2):
        path = os.path.join(HERE, "golden_ng32_izipx%d.npz" % izipx)
        np.savez_compressed(path, **make(izipx))
        print(path, os.path.getsize(path))
