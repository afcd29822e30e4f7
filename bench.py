#!/usr/bin/env python
"""Benchmark: particle-steps/s of the P3M KDK step (drift + PM1 + PM2 + PM3 + PP).

Default workload: 512^3 CDM particles in a 1000 Mpc/h box, fine mesh 1024^3
(PM1 256^3, PM2 64 tiles of 288^3, PM3 subtile meshes of 144^3 and up), int16
compressed coordinates, Zel'dovich ICs at z=49 (EH no-wiggle, A_s), reference
adaptive timestep.  One JSON line on rank 0.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload 512|128|proxy] [--deposit fixed|plain] [--graph on|off] [--pp queue|thread]
                  [--compare on|off] [--late on|off] [--full-run on|off] [--small on|off]

The headline is the chosen form (int64 fixed-point deposit, queue PP, each step one CUDA
graph) over K adaptive steps after W warm-up steps from z=49; the plain form (FP32 atomics,
thread-per-particle PP, eager launches) is timed in the same run over the same steps and
both are reported, with the relative P(k) difference of their final states.  On one GPU
the line also carries: the 512^3 run z=49 -> 0 in 100 steps in both forms (full_run), the
clustered 256^3 configuration evolved to z~0 (late_time), and the 128^3 configuration with
one oracle step on the host cores plus the adjoint's forward and backward (small_configs).

--impl reference times the CPU restatement of the reference path (oracle/, the
reference Fortran cannot be built here) on the host cores over a bounded sample of
the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cube_nu_b200 import cosmology  # noqa: E402
from cube_nu_b200.params import DEPOSIT_FIXED, DEPOSIT_FP32, config_512, config_late_256, config_plain_128  # noqa: E402

METRIC = "particle-steps/s P3M KDK @512^3"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}
# DRAM bytes (read + write) per class-2 PM3 box of 144^3, measured once with ncu on the
# proxy workload (one launch over 64 boxes) and kept here as constants: the 512^3 launch is
# too large to capture.  Traffic grows with the number of boxes, so a launch over B such
# boxes moves B times these.  The bench line labels the figure proxy_ncu_constant.
PM3_TRAFFIC_PER_BOX = {
    "deposit_pm3": (15048960 + 707247360) / 64,
    "fft_z_green_pm3": 1.910046e9 / 64,
    "fft_c2r_pm3": 1.485638e9 / 64,
}


def over_ranks(values, op: str, dist=None, device: str = "cuda"):
    """Elementwise max or sum of per-rank floats across the process group (identity
    without one).  Every rank must call it, with the same number of values."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(x) for x in t.tolist()]


def job_rate(total_particles: float, steps: int, seconds: float) -> float:
    """Whole-job particle-steps/s: every rank's particles over the slowest rank's time."""
    return total_particles * steps / seconds


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def workload(name: str):
    if name == "proxy":
        # same mesh sides as the 512^3 workload (PM2 288^3, PM3 144^3) on one tile: for ncu captures
        p = config_512()
        p.ng, p.nnt, p.box = 256, 1, 250.0
        return p, "proxy: 128^3 CDM, 250 Mpc/h, ng 256, one tile (PM2 288^3, PM3 64 subtiles 144^3), int16 ZIPX"
    if name == "512":
        p = config_512()
        desc = "512^3 CDM, 1000 Mpc/h, fine mesh 1024^3 (PM1 256^3, PM2 64x288^3, PM3 4096 subtiles), int16 ZIPX"
    else:
        p = config_plain_128()
        p.nic = 1
        desc = "128^3 CDM, 200 Mpc/h, fine mesh 256^3 (PM1 64^3, PM2 64x96^3, PM3 4096 subtiles), int8 ZIPX"
    return p, desc


# ------------------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ------------------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------
# algorithmic bytes per kernel launch (roofline numerators)
# ------------------------------------------------------------------------------------
def kernel_bytes(p, name: str, n_particles: int, napm, fixed: bool):
    """Algorithmic HBM bytes a kernel class must move over one whole step (all its
    launches together): mesh passes read and write each cell once at the element size
    of the pass, particle kernels read each particle's code and velocity once, the
    deposit adds 27 read-modify-writes per particle and box it lands in."""
    bx = 3 * p.izipx
    rb = 8 if fixed else 4

    def mesh(n, nbox, what, rb=rb):
        n3 = n ** 3 * nbox
        nh = n * n * (n // 2 + 1) * nbox
        return {"x": n3 * rb + nh * 8, "y": 2 * nh * 8, "z": 2 * nh * 8 + n * n * (n // 2 + 1) * 4,
                "c": nh * 8 + n3 * 4}[what]

    if name.startswith("fft_") and name.endswith("_pm3"):
        # all class-2 subtiles (the dominant class); the y pass runs forward and inverse
        n = p.nft(2)
        nb = int(napm[2]) if napm is not None else p.ns3
        what = {"fft_x_pm3": "x", "fft_y_pm3": "y", "fft_z_green_pm3": "z", "fft_c2r_pm3": "c"}[name]
        # the PM3 mesh is float in both deposit forms (the owner-computes fixed-point
        # deposit writes the converted sums)
        return mesh(n, nb, what, rb=4) * (2 if what == "y" else 1)
    if name.startswith("fft_") and name.endswith("_pm2"):
        what = {"fft_x_pm2": "x", "fft_y_pm2": "y", "fft_z_green_pm2": "z", "fft_c2r_pm2": "c"}[name]
        return mesh(p.ngt, p.ntiles, what) * (2 if what == "y" else 1)
    if name == "deposit_pm3" and fixed:
        # owner-computes form: every cell of every box written once as float (no memset,
        # no read-back), each particle's position code read once
        nbs = napm if napm is not None else [0, 0, p.ns3, 0, 0, 0]
        return int(sum(int(nbs[c]) * p.nft(c) ** 3 * 4 for c in range(2, 6)) + n_particles * bx)
    if name in ("deposit_pm1", "deposit_pm2", "deposit_pm3"):
        # read position code + cell index per particle, one read-modify-write of 27 cells
        boxes = {"deposit_pm1": 1.0, "deposit_pm2": (1 + 2 * p.ncb / p.nt) ** 3, "deposit_pm3": (1 + 2 / p.ntt) ** 3}[name]
        return int(n_particles * (bx + 4 + boxes * 27 * 2 * rb))
    if name in ("interp_pm1", "interp_pm2", "interp_pm3"):
        # position code + cell, velocity read+write, 27 force points x 3 (from phi)
        return int(n_particles * (bx + 4 + 24 + 27 * 4))
    if name == "pp":
        return int(n_particles * (bx + 4 + 24))
    if name in ("drift_dest",):
        return int(n_particles * (bx + 12 + 4 + 8 + 4 + 4))
    if name in ("drift_gather",):
        return int(n_particles * (2 * bx + 24 + 16 + 8))
    return None


# ------------------------------------------------------------------------------------
# CPU baseline (oracle on the host cores, bounded sample)
# ------------------------------------------------------------------------------------
def cpu_baseline(p, st, dt, dt_old, a_mid, vz, frac_tiles=1 / 64):
    """Time the oracle restatement on a bounded sample of the workload and scale it
    to one full step.  Returns (particle-steps/s, cores, sample description, seconds)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    O.set_threads(cores)
    xp, vp, pid, rhoc = st
    n = xp.shape[0]
    ntiles = p.ntiles
    tiles = max(1, int(round(ntiles * frac_tiles)))
    t0 = time.perf_counter()
    O.drift_sample(p, xp, vp, pid, rhoc, dt_old, dt, vz, tiles)
    t_drift = time.perf_counter() - t0
    v = vp.copy()
    t0 = time.perf_counter()
    out = O.kick(p, xp, v, rhoc, dt, a_mid, fixed=False, boxes_frac=tiles / ntiles)
    t_kick = time.perf_counter() - t0
    scale = ntiles / tiles
    t_full = t_drift * scale + out.t_pm1 + (out.t_pm2 + out.t_pm3 + out.t_pp) * scale
    sample = ("oracle FP32 restatement: drift of %d/%d tiles, PM1 full, PM2 %d/%d tiles, PM3+PP %d/%d subtiles; "
              "scaled to one full step (%.1f s measured)" % (tiles, ntiles, tiles, ntiles, tiles * p.nns ** 3,
                                                              p.ns3, t_drift + t_kick))
    return n / t_full, cores, sample, t_drift + t_kick


def make_ic(p, seed, device):
    """Host-side IC (numpy) for the CPU reference arm."""
    from cube_nu_b200 import ic

    d = ic.zeldovich(p, z_i=49.0, seed=seed)
    p.mass_p_cdm = d["mass_p_cdm"]
    return d


def device_ic(p, seed, device):
    """ICs generated on the GPU (cube_gpu_ic); returns the context and header values."""
    from cube_nu_b200 import ic
    from cube_nu_b200._lib import Context

    p.mass_p_cdm = float(p.ng) ** 3 / float(p.npglobal)
    ctx = Context(p, device=device)
    d = ic.zeldovich_device(ctx, p, z_i=49.0, seed=seed)
    return ctx, d


def pinned_like(a):
    import torch

    t = torch.empty(a.shape, dtype={np.int8: torch.int8, np.int16: torch.int16, np.float32: torch.float32,
                                    np.int64: torch.int64, np.int32: torch.int32}[a.dtype.type], pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out, t


def pinned_state(st):
    """Pinned host copies of a particle state (for the end-to-end leg)."""
    out = []
    for a in st:
        h, _ = pinned_like(a)
        out.append(h)
    return out


def run_form(p, args, local, dist, rank, replay=None, timed=True, want_base=False):
    """IC on the device, W warm-up steps and K timed steps of one form of the step.

    replay: the (dt, dt_old, a_mid, vz_max) of every step of another run, replayed here so
    both forms take the same steps; else the reference's adaptive timestep chooses them.
    Returns the timing, the per-kernel profile, the step inputs and outputs, the context
    (still open) and the state at the start of the timed steps when want_base."""
    import torch

    ctx, d = device_ic(p, seed=1 + rank, device=local)
    n = d["nplocal"]
    tab = cosmology.expansion_table(p.h0, p.omega_m, p.omega_r)
    bg = cosmology.Background.from_table(tab)
    S = cosmology.StepState(a=d["a"], dt_vmax=d["dt_vmax"], vz_max=d["vz_max"])
    bg.init_cursor(S.a)
    zck = [49.0, 0.0]
    steps_in = []

    def one_step(i):
        if replay is not None:
            dt, dt_old, a_mid, vz = replay[i]
        else:
            cosmology.timestep(bg, S, zck)
            dt, dt_old, a_mid, vz = S.dt, S.dt_old, S.a_mid, S.vz_max
        so = ctx.step(dt, dt_old, a_mid, vz)
        steps_in.append((dt, dt_old, a_mid, vz))
        S.dt_pm1, S.dt_pm2, S.dt_pm3, S.dt_pp, S.dt_vmax = so.dt_pm1, so.dt_pm2, so.dt_pm3, so.dt_pp, so.dt_vmax
        S.vz_max = so.vz_max
        return so

    for i in range(args.warmup):
        if i == args.warmup - 1:
            ctx.profile(True)  # a graph is captured with its timer events before the timed steps
        one_step(i)
    base = ctx.download() if want_base else None
    base_args = (S.dt, S.dt, S.a_mid, S.vz_max)
    ctx.profile(True)
    launches0 = ctx.launches()
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_wall = time.perf_counter()
    dev_ms = 0.0
    stage = np.zeros(7)
    sos = []
    for i in range(args.steps):
        so = one_step(args.warmup + i)
        dev_ms += so.tcat[6]
        stage += np.array(list(so.tcat)[:7])
        sos.append(so)
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    clk = clocks.stop()
    launches = ctx.launches() - launches0
    prof = ctx.profile_read()
    ctx.profile(False)
    dev_s, t_wall = over_ranks([dev_ms / 1e3, t_wall], "max", dist)
    return {"ctx": ctx, "n": n, "d": d, "S": S, "bg": bg, "zck": zck, "steps_in": steps_in, "sos": sos,
            "dev_s": dev_s, "t_wall": t_wall, "stage": stage, "clk": clk, "launches": launches, "prof": prof,
            "base": base, "base_args": base_args}


def late_leg(args, local, rank, z_late=0.05, max_evolve=2000, steps=5):
    """The clustered-PP configuration: 256^3 CDM in 100 Mpc/h (ng 256, 64 particles per
    coarse cell), evolved from z=49 in the chosen form to a checkpoint at z_late (outside
    any timed region), then `steps` steps toward z=0 timed in the chosen form and the same
    steps replayed by the plain form from the same state.  The evolution takes the
    reference's timestep with only its expansion and velocity limits (timestep.f90:20-34
    with the force criteria left out, ra_max = 0.1: about 40 steps), which still collapses
    the haloes (cells of ~10^4 particles); the timed steps use every criterion."""
    import torch

    from cube_nu_b200._lib import Context

    p = config_late_256()
    p.deposit_mode = DEPOSIT_FIXED
    p.step_graph = True
    p.pp_queue = True
    ctx, d = device_ic(p, seed=3 + rank, device=local)
    tab = cosmology.expansion_table(p.h0, p.omega_m, p.omega_r)
    bg = cosmology.Background.from_table(tab)
    S = cosmology.StepState(a=d["a"], dt_vmax=d["dt_vmax"], vz_max=d["vz_max"])
    bg.init_cursor(S.a)
    zck = [49.0, z_late]
    t0 = time.perf_counter()
    nev = 0

    def advance(evolve=False):
        if evolve:  # expansion and velocity limits only
            S.dt_pm1 = S.dt_pm2 = S.dt_pm3 = S.dt_pp = 1e3
        cosmology.timestep(bg, S, zck)
        si = (S.dt, S.dt_old, S.a_mid, S.vz_max)
        so = ctx.step(*si)
        S.dt_pm1, S.dt_pm2, S.dt_pm3, S.dt_pp, S.dt_vmax = so.dt_pm1, so.dt_pm2, so.dt_pm3, so.dt_pp, so.dt_vmax
        S.vz_max = so.vz_max
        return si, so

    while nev < max_evolve and not S.final_step:
        advance(evolve=True)
        nev += 1
    t_evolve = time.perf_counter() - t0
    # the timed steps head for z = 0 from the checkpoint at z_late
    zck.append(0.0)
    S.cur_checkpoint = len(zck)
    S.final_step = False
    state = ctx.download()
    res = {"workload": "256^3 CDM, 100 Mpc/h, ng 256 (64 particles per coarse cell), int16 ZIPX",
           "evolve_steps": nev, "evolve_s": round(t_evolve, 1), "a_start": S.a, "z_start": round(1 / S.a - 1, 4),
           "max_cell": int(state[3].max())}
    forms = {}
    replay = []
    ctx.profile(True)
    torch.cuda.synchronize()
    ms = 0.0
    pairs = cand = 0
    torch.cuda.nvtx.range_push("late_timed")  # lets a profiler pick these steps' launches
    for _ in range(steps):
        si, so = advance()
        replay.append(si)
        ms += so.tcat[6]
        pairs += so.pp_pairs
        cand += so.pp_candidates
    torch.cuda.nvtx.range_pop()
    prof = ctx.profile_read()
    forms["chosen"] = {"ms_per_step": round(ms / steps, 3), "value": round(state[0].shape[0] * steps / (ms / 1e3), 1),
                       "pp_ms_per_step": round(prof.get("pp", (0, 0))[0] / steps, 3),
                       "pm3_classes": list(so.napm)[2:6], "pp_pairs_per_step": pairs // steps,
                       "pp_candidates_per_step": cand // steps}
    ctx.close()
    q = config_late_256()
    q.deposit_mode = DEPOSIT_FP32
    q.mass_p_cdm = p.mass_p_cdm
    with Context(q, device=local) as c2:
        c2.upload(*state)
        c2.profile(True)
        ms = 0.0
        for si in replay:
            so = c2.step(*si)
            ms += so.tcat[6]
        prof = c2.profile_read()
    forms["plain"] = {"ms_per_step": round(ms / steps, 3), "value": round(state[0].shape[0] * steps / (ms / 1e3), 1),
                      "pp_ms_per_step": round(prof.get("pp", (0, 0))[0] / steps, 3)}
    forms["chosen_over_plain"] = round(forms["plain"]["ms_per_step"] / forms["chosen"]["ms_per_step"], 4)
    res["forms"] = forms
    res["steps"] = steps
    return res


def full_run_leg(args, local, rank, nsteps=100):
    """The 512^3 configuration as its run is defined: 512^3 CDM in 1000 Mpc/h from the
    z=49 Zel'dovich ICs to z=0 in `nsteps` KDK steps of equal code time
    (cosmology.fixed_steps, with the closing half drift at z=0), once in the chosen form and
    once in the plain form from the same ICs.  Per form: the device time of every step (the
    library's step events; the chosen form's PP tuning and graph captures run between
    steps), the wall time of the whole run, the per-stage split, the occupancy the run
    reaches, and the P(k) of the final particles on the 1024^3 grid; the two spectra are
    compared for k < k_Nyq/2."""
    import torch

    nw = None
    forms = {}
    xis = {}
    # plain_repeat: the plain form once more from the same ICs; its FP32 atomics sum in a
    # different order, so its P(k) against the first plain run measures how far rounding
    # differences alone carry the particles apart over the run
    for form in ("chosen", "plain", "plain_repeat"):
        q = config_512()
        fixed = form == "chosen"
        q.deposit_mode = DEPOSIT_FIXED if fixed else DEPOSIT_FP32
        q.step_graph = fixed
        q.pp_queue = fixed and (q.izipx == 1 or q.nt < 127)
        nw = pk_grid(q)
        ctx, d = device_ic(q, seed=1 + rank, device=local)
        tab = cosmology.expansion_table(q.h0, q.omega_m, q.omega_r)
        bg = cosmology.Background.from_table(tab)
        sched = cosmology.fixed_steps(bg, d["a"], 1.0, nsteps)
        vz = d["vz_max"]
        ctx.profile(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        per = []
        stage = np.zeros(7)
        stage_first = np.zeros(7)
        pairs = cand = 0
        q10 = max(1, nsteps // 10)
        for i, (dt, dt_old, a_mid, _) in enumerate(sched):
            so = ctx.step(dt, dt_old, a_mid, vz)
            vz = so.vz_max
            per.append(so.tcat[6])
            stage += np.array(list(so.tcat)[:7])
            if i < q10:
                stage_first += np.array(list(so.tcat)[:7])
            pairs += so.pp_pairs
            cand += so.pp_candidates
        ctx.drift(sched[-1][0], 0.0, vz)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        ctx.profile(False)
        n = d["nplocal"]
        st = ctx.download()
        xis[form] = ctx.power(nw, n_corr=0)[0]
        ctx.close()
        if form == "plain_repeat":
            continue
        dev_s = sum(per) / 1e3
        forms[form] = {"value": round(n * nsteps / dev_s, 1), "ms_per_step": round(sum(per) / nsteps, 3),
                       "wall_s": round(wall, 2),
                       "ms_per_step_first_last_tenth": [round(float(np.mean(per[:q10])), 3),
                                                        round(float(np.mean(per[-q10:])), 3)],
                       "ms_first_steps": [round(float(x), 2) for x in per[:q10]],
                       "stage_ms_per_step": {k: round(float(v) / nsteps, 3) for k, v in
                                             zip(("drift", "pm1", "pm2", "pm3", "pp", "kick", "step"), stage)},
                       "stage_ms_per_step_first_tenth": {k: round(float(v) / q10, 3) for k, v in
                                                         zip(("drift", "pm1", "pm2", "pm3", "pp", "kick", "step"),
                                                             stage_first)},
                       "pm3_classes_end": list(so.napm)[2:6], "max_cell_end": int(st[3].max()),
                       "pp_pairs_per_step": pairs // nsteps, "pp_candidates_per_step": cand // nsteps,
                       "deposit": "int64 fixed-point" if fixed else "fp32 atomics", "graph": fixed,
                       "pp": "queue" if q.pp_queue else "thread"}
    knyq = math.pi * nw / 1000.0
    b = xis["plain"]

    def dpp(x, kmax):
        sel = (b[:, 0] > 0) & (b[:, 1] > 0) & (b[:, 1] < kmax)
        return float(np.abs(x[sel, 2] / b[sel, 2] - 1).max())

    forms["chosen_over_plain"] = round(forms["plain"]["ms_per_step"] / forms["chosen"]["ms_per_step"], 4)
    return {"workload": "512^3 CDM, 1000 Mpc/h, ng 1024, int16 ZIPX, z=49 -> 0 in %d equal code-time KDK steps" % nsteps,
            "steps": nsteps, "forms": forms, "pk_grid": nw, "k_nyq_hmpc": round(knyq, 4),
            "dP_over_P_max": {"chosen_vs_plain_k_lt_knyq_2": dpp(xis["chosen"], knyq / 2),
                              "chosen_vs_plain_k_lt_knyq_4": dpp(xis["chosen"], knyq / 4),
                              "plain_repeat_vs_plain_k_lt_knyq_2": dpp(xis["plain_repeat"], knyq / 2),
                              "plain_repeat_vs_plain_k_lt_knyq_4": dpp(xis["plain_repeat"], knyq / 4)}}


def small_configs_leg(args, local, rank, cpu=True):
    """The two smaller configurations of the benchmark set at full size.
    128^3: 128^3 CDM in 200 Mpc/h, ng 256, int8 ZIPX, PP on, z=49 -> 10 in 10 equal
    code-time KDK steps from the device ICs, in both forms (device time per step); and,
    when cpu, one whole step of the oracle in FP32 on all host cores from the same state
    (a measured step, not a sample scaled up).
    adjoint: 128^3 particles on a 256^3 mesh in 256 Mpc/h, PM only, 20 KDK steps z=20 -> 0,
    loss = mean squared difference of the final TSC density from a second seed's, gradient
    with respect to the 128^3 white-noise modes by the hand-written adjoint with a checkpoint
    every 5 steps; forward and backward timed on the device (the third evaluation of
    three)."""
    import torch

    from cube_nu_b200 import adjoint as A
    from cube_nu_b200.params import config_plain_128

    out = {}
    forms = {}
    state = None
    for form in ("chosen", "plain"):
        q = config_plain_128()
        q.nic = 1
        fixed = form == "chosen"
        q.deposit_mode = DEPOSIT_FIXED if fixed else DEPOSIT_FP32
        q.step_graph = fixed
        q.pp_queue = fixed
        ctx, d = device_ic(q, seed=1 + rank, device=local)
        tab = cosmology.expansion_table(q.h0, q.omega_m, q.omega_r)
        bg = cosmology.Background.from_table(tab)
        sched = cosmology.fixed_steps(bg, d["a"], 1 / 11.0, 10)
        vz = d["vz_max"]
        if state is None:
            state = (ctx.download(), sched, vz, q)
        ctx.profile(True)
        ms = 0.0
        for dt, dt_old, a_mid, _ in sched:
            so = ctx.step(dt, dt_old, a_mid, vz)
            vz = so.vz_max
            ms += so.tcat[6]
        ctx.profile(False)
        n = d["nplocal"]
        ctx.close()
        forms[form] = {"ms_per_step": round(ms / len(sched), 3), "value": round(n * len(sched) / (ms / 1e3), 1)}
    forms["chosen_over_plain"] = round(forms["plain"]["ms_per_step"] / forms["chosen"]["ms_per_step"], 4)
    out["config_128"] = {"workload": "128^3 CDM, 200 Mpc/h, ng 256, int8 ZIPX, z=49 -> 10 in 10 KDK steps",
                         "forms": forms}
    if cpu:
        from oracle import oracle as O

        (xp, vp, pid, rhoc), sched, vz, q = state
        cores = os.cpu_count() or 1
        O.set_threads(cores)
        dt, dt_old, a_mid, _ = sched[0]
        t0 = time.perf_counter()
        xp2, vp2, pid2, rhoc2 = O.drift(q, xp, vp, pid, rhoc, dt_old, dt, vz)
        O.kick(q, xp2, vp2, rhoc2, dt, a_mid, fixed=False)
        secs = time.perf_counter() - t0
        out["config_128"]["cpu_oracle"] = {"value": round(xp.shape[0] / secs, 1), "unit": "particle-steps/s",
                                           "cores": cores, "kind": "port",
                                           "sample": "one whole step (drift + kick with PM1, PM2, PM3, PP) of "
                                                     "the oracle in FP32, first step of the run",
                                           "seconds": round(secs, 2)}
    # the adjoint
    p = config_plain_128()
    p.box = 256.0
    n, n_lat, m = 256, 128, 8.0
    steps, d_close = A.kdk_schedule(p, 20.0, 0.0, 20)
    a0 = 1 / 21.0
    dpm = A.DPM(n, 1.5, m, device=local)
    op = A.ic_operator(p, n_lat, a0)
    gen = torch.Generator(device="cuda").manual_seed(11)
    w = torch.randn((n_lat,) * 3, generator=gen, device="cuda")
    w2 = torch.randn((n_lat,) * 3, generator=gen, device="cuda")
    with torch.no_grad():
        x0, v0 = A.zeldovich(w2, p, a0, op)
        target = dpm.density(A.Simulate.apply(x0.contiguous(), v0.contiguous(), dpm, steps, d_close, 5))
    fw = bw = 0.0
    for _ in range(3):
        wg = w.clone().requires_grad_(True)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        loss = A.density_loss(wg, target, dpm, p, a0, steps, d_close, every=5, op=op)
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        fw, bw = e0.elapsed_time(e1), e1.elapsed_time(e2)
    dpm.close()
    np3 = n_lat ** 3
    out["adjoint"] = {"workload": "128^3 particles, mesh 256^3, 256 Mpc/h, PM only, 20 KDK steps z=20 -> 0, "
                                  "density MSE loss, gradient w.r.t. the 128^3 noise modes, checkpoint every 5",
                      "forward_ms": round(fw, 2), "backward_ms": round(bw, 2),
                      "forward_particle_steps_per_s": round(np3 * 20 / (fw / 1e3), 1),
                      "gradient_particle_steps_per_s": round(np3 * 20 / ((fw + bw) / 1e3), 1)}
    return out


def pk_grid(p):
    """cicpower grid of the precision check: 2*ng as utilities/Makefile's FFTFINE builds it,
    capped at 1024^3 (the 512^3 workload's 2048^3 grid would hold ~100 GB beside the step)."""
    return min(2 * p.ng, 1024)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="512", choices=["512", "128", "proxy", "late"],
                    help="late: only the clustered 256^3 configuration evolved to z~0 (its own JSON line)")
    ap.add_argument("--deposit", default="fixed", choices=["fixed", "plain"])
    ap.add_argument("--graph", default="on", choices=["on", "off"],
                    help="replay each step as one captured CUDA graph (cube_params.step_graph)")
    ap.add_argument("--pp", default="queue", choices=["queue", "thread"],
                    help="PP as the autotuned cell work queue (cube_params.pp_queue) or a thread per particle")
    ap.add_argument("--compare", default="on", choices=["on", "off"],
                    help="also time the plain form (FP32 atomics, eager) over the same steps")
    ap.add_argument("--late", default="on", choices=["on", "off"],
                    help="also time the clustered-PP configuration (256^3, 100 Mpc/h) evolved to z~0, both forms")
    ap.add_argument("--small", default="on", choices=["on", "off"],
                    help="also time the 128^3 configuration (both forms, and one oracle step) and the adjoint")
    ap.add_argument("--full-run", default="on", choices=["on", "off"],
                    help="also run the 512^3 configuration z=49 -> 0 in 100 KDK steps, both forms")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-json", default="")
    ap.add_argument("--pk", type=int, default=0,
                    help="after the timed steps, also time cube_gpu_power on an NW^3 mesh (outside the metric)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    p, desc = workload(args.workload)
    fixed = args.deposit == "fixed"
    p.deposit_mode = DEPOSIT_FIXED if fixed else DEPOSIT_FP32
    p.step_graph = args.graph == "on"
    p.pp_queue = args.pp == "queue" and (p.izipx == 1 or p.nt < 127)

    import torch

    if args.impl == "reference":
        if rank != 0:
            return 0
        run_reference(args, p, desc)
        return 0

    torch.cuda.set_device(local)
    if args.workload == "late":
        if rank == 0:
            print(json.dumps({"late_time": late_leg(args, local, rank)}), flush=True)
        return 0
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    R = run_form(p, args, local, dist, rank, want_base=(rank == 0 and not args.no_cpu_baseline))
    ctx, n, S, bg, zck = R["ctx"], R["n"], R["S"], R["bg"], R["zck"]
    total_particles = over_ranks([n], "sum", dist)[0]
    value = job_rate(total_particles, args.steps, R["dev_s"])
    nw = pk_grid(p)
    xi_chosen = ctx.power(nw, n_corr=0)[0]

    # ---------------- end to end through the C ABI with pinned host buffers ----------------
    xh, vh, ph, rh = pinned_state(ctx.download())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_e2e = time.perf_counter()
    for _ in range(args.steps):
        # host-resident state: cube_gpu_step_host uploads it from the pinned arrays, steps,
        # and writes the new state back (copies the step does not wait for overlap it)
        cosmology.timestep(bg, S, zck)
        so = ctx.step_host(xh, vh, ph, rh, S.dt, S.dt_old, S.a_mid, S.vz_max)
        S.dt_pm1, S.dt_pm2, S.dt_pm3, S.dt_pp, S.dt_vmax = so.dt_pm1, so.dt_pm2, so.dt_pm3, so.dt_pp, so.dt_vmax
        S.vz_max = so.vz_max
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t_e2e
    t_e2e = over_ranks([t_e2e], "max", dist)[0]
    io_bytes = n * (3 * p.izipx + 12 + 8) + p.ncells * 4
    e2e_value = job_rate(total_particles, args.steps, t_e2e)

    analysis = None
    if args.pk:
        # power spectrum of the evolved particles (cicpower + auto_power): first call
        # builds the FFT tables, the second is timed on the device
        ctx.power(args.pk, n_corr=1)
        xi, _, po = ctx.power(args.pk)
        analysis = {"pk_nw": args.pk, "pk_ms": round(po.ms, 3), "pk_alpha": float(po.alpha),
                    "pk_corrections": po.n_corr_done, "pk_nbin": int(po.nbin)}
    ctx.close()

    # ---------------- the plain form over the same steps ----------------
    plain = None
    if args.compare == "on" and (fixed or p.step_graph or p.pp_queue):
        q, _ = workload(args.workload)
        q.deposit_mode = DEPOSIT_FP32
        q.step_graph = False
        q.pp_queue = False
        P = run_form(q, args, local, dist, rank, replay=R["steps_in"])
        xi_plain = P["ctx"].power(nw, n_corr=0)[0]
        P["ctx"].close()
        plain = {"value": job_rate(total_particles, args.steps, P["dev_s"]),
                 "ms_per_step": P["dev_s"] * 1e3 / args.steps, "xi": xi_plain,
                 "stage": P["stage"] / args.steps}

    late = None
    if args.late == "on" and args.workload == "512" and world == 1:
        late = late_leg(args, local, rank)
    small = None
    if args.small == "on" and args.workload == "512" and world == 1:
        try:
            small = small_configs_leg(args, local, rank, cpu=not args.no_cpu_baseline)
        except Exception as e:  # reported in the line; the headline above stands
            small = {"error": str(e)[:300]}
    full = None
    if args.full_run == "on" and args.workload == "512" and world == 1:
        try:
            full = full_run_leg(args, local, rank)
        except Exception as e:  # reported in the line; the headline above stands
            full = {"error": str(e)[:300]}

    if rank == 0:
        peaks, peak_kind = load_peaks()
        sos = R["sos"]
        napm = list(sos[-1].napm)
        prof = R["prof"]
        # roofline of the dominant kernel class
        rows = []
        for name, (ms, cnt) in prof.items():
            if cnt == 0:
                continue
            b = kernel_bytes(p, name, n, napm, fixed)  # algorithmic bytes of the whole step's work
            per_step_ms = ms / args.steps
            rows.append((ms, name, cnt, ms / cnt, b, per_step_ms))
        rows.sort(reverse=True)
        dom = next((r for r in rows if r[4] is not None), None)
        hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
        roof = None
        if dom:
            launches_per_step = dom[2] / args.steps
            ach = dom[4] / (dom[5] / 1e3) / 1e9
            traffic = None
            if dom[1] in PM3_TRAFFIC_PER_BOX and p.nft(2) == 144 and sum(napm[3:6]) == 0:
                traffic = int(PM3_TRAFFIC_PER_BOX[dom[1]] * napm[2] / launches_per_step)
            roof = {"kernel": dom[1], "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(ach / hbm, 4), "traffic": traffic,
                    "traffic_source": ("proxy_ncu_constant: ncu DRAM bytes of one 64-box launch of the proxy "
                                       "workload, scaled by boxes (not measured in this run)" if traffic else None),
                    "peak_kind": peak_kind, "avg_launch_ms": round(dom[3], 4),
                    "launches_per_step": launches_per_step,
                    "algorithmic_bytes_per_launch": int(dom[4] / launches_per_step)}
        # PP on the FP32 pipe: 9 flops per candidate pair (dx 3, r^2 5, compare 1) and 35 more
        # per pair within range (sqrt, divide, two degree-6 F_ra, scale, accumulate)
        pp = None
        pp_ms, pp_n = prof.get("pp", (0.0, 0))
        if pp_n:
            cand = sum(int(so.pp_candidates) for so in sos)
            pairs = sum(int(so.pp_pairs) for so in sos)
            flops = 9.0 * cand + 35.0 * pairs
            mhz = R["clk"].get("sm_mhz") or 1965.0
            fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12  # TFLOP/s at the sampled SM clock
            tf = flops / (pp_ms / 1e3) / 1e12
            pp = {"tflops": round(tf, 3), "fp32_peak_tflops": round(fp32_peak, 1), "frac": round(tf / fp32_peak, 4),
                  "candidates_per_step": cand // args.steps, "pairs_per_step": pairs // args.steps,
                  "ms_per_step": round(pp_ms / args.steps, 3)}
        cpu = None
        if R["base"] is not None:
            v, cores, sample, secs = cpu_baseline(p, R["base"], *R["base_args"])
            cpu = {"value": round(v, 1), "unit": "particle-steps/s", "cores": cores, "kind": "port",
                   "sample": sample, "sample_seconds": round(secs, 2), "extrapolated_to_full_step": True}
        forms = {"chosen": {"value": round(value, 1), "ms_per_step": round(R["dev_s"] * 1e3 / args.steps, 3),
                            "deposit": "int64 fixed-point" if fixed else "fp32 atomics",
                            "graph": bool(p.step_graph), "pp": "queue" if p.pp_queue else "thread"}}
        precision = None
        if plain:
            forms["plain"] = {"value": round(plain["value"], 1), "ms_per_step": round(plain["ms_per_step"], 3),
                              "deposit": "fp32 atomics", "graph": False, "pp": "thread",
                              "stage_ms_per_step": {k: round(float(v), 3) for k, v in
                                                    zip(("drift", "pm1", "pm2", "pm3", "pp", "kick", "step"),
                                                        plain["stage"])}}
            forms["chosen_over_plain"] = round(value / plain["value"], 4)
            a, b = xi_chosen, plain["xi"]
            knyq = math.pi * nw / p.box
            sel = (b[:, 0] > 0) & (b[:, 1] > 0) & (b[:, 1] < knyq / 2)
            rel = np.abs(a[sel, 2] / b[sel, 2] - 1)
            precision = {"dP_over_P_max_chosen_vs_plain": float(rel.max()), "bins": int(sel.sum()),
                         "grid": nw, "k_max_hmpc": round(knyq / 2, 4),
                         "note": "both forms after the same steps; against the FP64 oracle see tests/test_precision.py"}
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(R["dev_s"] * 1e3 / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (Zel'dovich ICs z=49, EH no-wiggle, seeded)",
            "config": {"workload": desc, "particles_per_gpu": n, "ng": p.ng, "box": p.box,
                       "deposit": "int64 fixed-point" if fixed else "fp32 atomics",
                       "step_graph": bool(p.step_graph), "pp": "queue" if p.pp_queue else "thread",
                       "timestep": "reference adaptive (timestep.f90)", "parallelism": "replicas x%d" % world,
                       "l2": "inputs larger than L2 (%.1f GB particle state)" % (n * 26 / 1e9),
                       "pm3_classes": napm[2:6], "a_end": R["S"].a},
            "e2e": {"value": round(e2e_value, 1), "unit": "particle-steps/s", "h2d_bytes_per_step": io_bytes,
                    "d2h_bytes_per_step": io_bytes},
            "gpu_launches": int(R["launches"]),
            "roofline": roof,
            "pp_fp32": pp,
            "forms": forms,
            "precision": precision,
            "cpu_baseline": cpu,
            "clocks": R["clk"],
            "wall_s": round(R["t_wall"], 3),
            "stage_ms_per_step": {k: round(float(v) / args.steps, 3) for k, v in
                                  zip(("drift", "pm1", "pm2", "pm3", "pp", "kick", "step"), R["stage"])},
            "mass_check": {"pm1": sos[-1].mass_pm1, "pm2": sos[-1].mass_pm2, "pm3": sos[-1].mass_pm3,
                           "particles": n},
        }
        if late:
            line["late_time"] = late
        if full:
            line["full_run"] = full
        if small:
            line["small_configs"] = small
        if analysis:
            line["analysis"] = analysis
        if args.profile_json:
            with open(args.profile_json, "w") as f:
                json.dump({"kernels": [{"name": r[1], "total_ms": r[0], "launches": r[2], "avg_ms": r[3],
                                        "alg_bytes_per_step": r[4], "ms_per_step": r[5]} for r in rows],
                           "steps": args.steps}, f, indent=1)
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_reference(args, p, desc):
    """--impl reference: the CPU restatement timed on the host cores."""
    import torch

    if torch.cuda.is_available():
        # the same ICs as the GPU arm, generated on the device and copied to the host
        ctx, d = device_ic(p, seed=1, device=0)
        st = ctx.download()
        ctx.close()
    else:
        d = make_ic(p, seed=1, device=None)
        st = (d["xp"], d["vp"], d["pid"], d["rhoc"])
    n = st[0].shape[0]
    tab = cosmology.expansion_table(p.h0, p.omega_m, p.omega_r)
    bg = cosmology.Background.from_table(tab)
    S = cosmology.StepState(a=d["a"], dt_vmax=d["dt_vmax"], vz_max=d["vz_max"])
    bg.init_cursor(S.a)
    cosmology.timestep(bg, S, [49.0, 0.0])
    rates = []
    cores = os.cpu_count() or 1
    sample = ""
    for i in range(args.warmup + args.steps):
        v, cores, sample, secs = cpu_baseline(p, st, S.dt, S.dt_old, S.a_mid, S.vz_max)
        if i >= args.warmup:
            rates.append(v)
        if i == 0 and secs * (args.warmup + args.steps) > 240:
            # keep the whole run within a few minutes: one warm-up, one timed sample
            args.warmup, args.steps = 0, 1
            rates.append(v)
            break
    value = float(np.mean(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": "particle-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(n / value * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (Zel'dovich ICs z=49, EH no-wiggle, seeded)",
        "config": {"workload": desc, "particles_per_gpu": n, "ng": p.ng, "box": p.box,
                   "timestep": "reference adaptive (timestep.f90)",
                   "reference": "CPU restatement of the reference Fortran path (gfortran/FFTW absent)"},
        "cpu_baseline": {"value": round(value, 1), "unit": "particle-steps/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 1), "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    sys.exit(main())
