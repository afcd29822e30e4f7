"""Host driver mirroring CUBE's main program for one image (main.f90:13-61).

    initialize -> particle_initialization -> loop {timestep; drift; kick; at a
    checkpoint: drift(dt_old=0), checkpoint} -> finalize

The step itself runs on the GPU through the C ABI (cube_gpu_step); the timestep
(timestep.f90) and checkpoint I/O (checkpoint.f90) stay on the host, as a Fortran host
keeps them.  Stage times go into a tcat-like table (basic_functions.f08:20-35):
column 2 drift, 11 PM1, 12 PM2, 13 PM3, 14 PP, 100 whole step.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

from . import checkpoint as ckio
from . import cosmology
from ._lib import Context
from .params import Params


@dataclasses.dataclass
class StepRecord:
    timestep: int
    a: float
    z: float
    dt: float
    dt_pm1: float
    dt_pm2: float
    dt_pm3: float
    dt_pp: float
    dt_vmax: float
    napm: list
    tcat_ms: dict


class Simulation:
    """One image of CUBE's time loop on the GPU."""

    def __init__(self, params: Params, z_checkpoint: list[float], device: int = 0, opath: str | None = None):
        self.p = params
        self.z_checkpoint = list(z_checkpoint)
        self.opath = opath
        self.ctx = Context(params, device=device)
        tab = cosmology.expansion_table(params.h0, params.omega_m, params.omega_r)
        self.bg = cosmology.Background.from_table(tab)
        self.state: cosmology.StepState | None = None
        self.history: list[StepRecord] = []
        self.header = None

    # particle_initialization.f90
    def load(self, xp, vp, pid, rhoc, a: float, dt_vmax: float = 1e3, vz_max: float = 0.0, header=None):
        self.ctx.upload(xp, vp, pid, rhoc)
        self.state = cosmology.StepState(a=a, dt_vmax=dt_vmax, vz_max=vz_max)
        self.bg.init_cursor(a)
        self.header = header

    def load_checkpoint(self, z: float):
        ck = ckio.read(self.opath, 1, z, self.p.izipx)
        h = ck.header
        self.p.mass_p_cdm = float(h["mass_p_cdm"])
        self.load(ck.xp, ck.vp, ck.pid, ck.rhoc, a=1.0 / (1.0 + z), dt_vmax=float(h["dt_vmax"]) or 1e3,
                  vz_max=float(h["vz_max"]), header=h)
        st = self.state
        st.timestep = int(h["timestep"])
        st.t, st.tau = float(h["t"]), float(h["tau"])
        for k in ("dt_pm1", "dt_pm2", "dt_pm3", "dt_pp"):
            v = float(h[k])
            setattr(st, k, v if v > 0 else 1e3)

    def step(self) -> StepRecord:
        """One loop body of main.f90:30-59 (timestep, drift, kick; checkpoint handling)."""
        st = self.state
        cosmology.timestep(self.bg, st, self.z_checkpoint)
        so = self.ctx.step(st.dt, st.dt_old, st.a_mid, st.vz_max)
        st.dt_pm1, st.dt_pm2, st.dt_pm3, st.dt_pp = so.dt_pm1, so.dt_pm2, so.dt_pm3, so.dt_pp
        st.dt_vmax, st.vz_max = so.dt_vmax, so.vz_max
        rec = StepRecord(st.timestep, st.a, 1.0 / st.a - 1.0, st.dt, so.dt_pm1, so.dt_pm2, so.dt_pm3, so.dt_pp,
                         so.dt_vmax, list(so.napm),
                         {2: so.tcat[0], 11: so.tcat[1], 12: so.tcat[2], 13: so.tcat[3], 14: so.tcat[4],
                          100: so.tcat[6]})
        self.history.append(rec)
        if st.checkpoint_step:
            # closing half drift with dt_old=0 (main.f90:39-41), then write
            # (the next timestep sets dt_old=dt again, timestep.f90:11, as in the reference)
            self.ctx.drift(st.dt, 0.0, st.vz_max)
            if self.opath:
                self.write_checkpoint(self.z_checkpoint[st.cur_checkpoint - 1])
            st.cur_checkpoint += 1
        return rec

    def run(self, max_steps: int = 100000) -> list[StepRecord]:
        for _ in range(max_steps):
            self.step()
            if self.state.final_step and self.state.checkpoint_step:
                break
        return self.history

    def write_checkpoint(self, z: float):
        xp, vp, pid, rhoc = self.ctx.download()
        st = self.state
        h = ckio.new_header(
            nplocal=xp.shape[0], npglobal=xp.shape[0], izipx=self.p.izipx, izipv=2, image=1, nn=1, nnt=self.p.nnt,
            nt=self.p.nt, ncell=self.p.nc, ncb=self.p.ncb, timestep=st.timestep, cur_checkpoint=st.cur_checkpoint,
            a=st.a, t=st.t, tau=st.tau, dt_pp=st.dt_pp, dt_pm3=st.dt_pm3, dt_pm2=st.dt_pm2, dt_pm1=st.dt_pm1,
            dt_vmax=st.dt_vmax, mass_p_cdm=self.p.particle_mass(), box=self.p.box, h0=self.p.h0,
            omega_m=self.p.omega_m, omega_l=self.p.omega_l, z_i=self.z_checkpoint[0], vz_max=st.vz_max,
            vsim2phys=(1.5 / st.a) * self.p.box * 100.0 * np.sqrt(self.p.omega_m) / self.p.ng)
        ckio.write(self.opath, 1, z, ckio.Checkpoint(h, xp, vp, rhoc, pid))

    def close(self):
        self.ctx.close()
