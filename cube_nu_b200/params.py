"""Run parameters, mirroring CUBE's ``parameters.f90``.

The Fortran reference fixes these as compile-time ``parameter`` constants
(parameters.f90:8-133).  Here they are a dataclass that is converted to the C
struct ``cube_params`` of ``include/cube_gpu.h``; derived sizes follow
parameters.f90:57-82.
"""
from __future__ import annotations

import ctypes
import dataclasses

RATIO_SF = (0, 1, 2, 4, 6, 8, 12, 16)  # parameters.f90:26, 1-based (index 0 unused)

DEPOSIT_FP32 = 0
DEPOSIT_FIXED = 1


class CParams(ctypes.Structure):
    """ctypes mirror of ``cube_params`` (include/cube_gpu.h)."""

    _fields_ = [
        ("ng", ctypes.c_int64),
        ("ratio_cs", ctypes.c_int64),
        ("nnt", ctypes.c_int64),
        ("nns", ctypes.c_int64),
        ("np_nc", ctypes.c_int64),
        ("ncb", ctypes.c_int64),
        ("ngb", ctypes.c_int64),
        ("izipx", ctypes.c_int32),
        ("pm3_on", ctypes.c_int32),
        ("pp_on", ctypes.c_int32),
        ("deposit_mode", ctypes.c_int32),
        ("box", ctypes.c_float),
        ("app", ctypes.c_float),
        ("apm1c", ctypes.c_float),
        ("apm2", ctypes.c_float),
        ("apm3f", ctypes.c_float),
        ("mass_p_cdm", ctypes.c_float),
        ("f_nu", ctypes.c_float),
        ("np_capacity", ctypes.c_int64),
        ("max_segment", ctypes.c_int32),
        ("step_graph", ctypes.c_int32),
        ("pp_queue", ctypes.c_int32),
        ("nslab", ctypes.c_int32),
        ("slab", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 3),
    ]


@dataclasses.dataclass
class Params:
    """One image's geometry and physics switches (parameters.f90 names)."""

    ng: int = 128            # fine cells per dimension (parameters.f90:24)
    ratio_cs: int = 4        # fine cells per coarse cell (:25)
    nnt: int = 4             # tiles per dimension (:28)
    nns: int = 4             # subtiles per tile per dimension (:29)
    np_nc: int = 4           # particles per coarse cell per dimension (:32)
    ncb: int = 4             # coarse ghost depth (:81)
    ngb: int = 16            # PM2 buffer, fine cells (:61)
    nic: int = 2             # IC grid refinement (:33)
    izipx: int = 2           # bytes per compressed coordinate (:10)
    pm3_on: bool = True      # kick.f90:9
    pp_on: bool = True       # kick.f90:10
    deposit_mode: int = DEPOSIT_FP32
    box: float = 600.0       # Mpc/h (:23)
    app: float = 0.06        # PP softening, fine cells (:46)
    apm1c: float = 3.5       # (:38)
    apm2: float = 3.5        # (:40)
    apm3f: float = 3.5       # (:42)
    mass_p_cdm: float = 0.0  # 0: derive ng^3/npglobal (ic.f90:839)
    f_nu: float = 0.0
    np_capacity: int = 0
    max_segment: int = 0
    step_graph: bool = False  # cube_gpu_step replays each step as one captured CUDA graph
    pp_queue: bool = False    # PP as an autotuned work queue over cells (chosen form)
    nslab: int = 1            # z-slabs of tile layers the box is split into, one rank each
    slab: int = 0             # this rank's slab
    # cosmology (parameters.f90:101-125; values of the benchmark configs)
    h0: float = 0.6817
    omega_c: float = 0.2532
    omega_b: float = 0.0481
    omega_r: float = 5.046734693877551e-05
    n_s: float = 0.9693
    A_s: float = 2.122e-09

    # ---- derived sizes (parameters.f90:57-82) ----
    @property
    def nc(self) -> int:
        return self.ng // self.ratio_cs

    @property
    def nt(self) -> int:
        return self.nc // self.nnt

    @property
    def ntt(self) -> int:
        return self.nt // self.nns

    @property
    def ngp(self) -> int:
        return self.ng // self.nnt

    @property
    def ngt(self) -> int:
        return self.ngp + 2 * self.ngb

    def nfp(self, iapm: int) -> int:
        return (self.ngp // self.nns) * RATIO_SF[iapm]

    def nfb(self, iapm: int) -> int:
        return self.ratio_cs * RATIO_SF[iapm]

    def nft(self, iapm: int) -> int:
        return self.nfp(iapm) + 2 * self.nfb(iapm)

    @property
    def npglobal(self) -> int:
        return (self.nc * self.np_nc) ** 3

    @property
    def ntiles(self) -> int:
        return self.nnt ** 3

    @property
    def ns3(self) -> int:
        return (self.nnt * self.nns) ** 3

    @property
    def ncells(self) -> int:
        return self.nc ** 3

    @property
    def omega_m(self) -> float:
        return self.omega_c + self.omega_b

    @property
    def omega_l(self) -> float:
        return 1.0 - self.omega_m - self.omega_r

    @property
    def xdtype(self):
        import numpy as np

        return np.int8 if self.izipx == 1 else np.int16

    def particle_mass(self) -> float:
        if self.mass_p_cdm > 0:
            return self.mass_p_cdm
        return float(self.ng) ** 3 / float(self.npglobal)

    def validate(self) -> None:
        if self.ng % self.ratio_cs or self.nc % self.nnt or self.nt % self.nns:
            raise ValueError("ng, nnt, nns must divide evenly (parameters.f90:57-59)")
        if self.izipx not in (1, 2):
            raise ValueError("izipx must be 1 or 2")
        if self.nt < self.ncb:
            raise ValueError("tiles must be at least ncb coarse cells wide")
        if self.nslab < 1 or self.nnt % self.nslab or not 0 <= self.slab < self.nslab:
            raise ValueError("nslab must divide nnt, and 0 <= slab < nslab")

    def to_c(self) -> CParams:
        self.validate()
        return CParams(
            ng=self.ng, ratio_cs=self.ratio_cs, nnt=self.nnt, nns=self.nns, np_nc=self.np_nc,
            ncb=self.ncb, ngb=self.ngb, izipx=self.izipx, pm3_on=int(self.pm3_on),
            pp_on=int(self.pp_on), deposit_mode=int(self.deposit_mode), box=self.box, app=self.app,
            apm1c=self.apm1c, apm2=self.apm2, apm3f=self.apm3f,
            mass_p_cdm=self.particle_mass(), f_nu=self.f_nu, np_capacity=self.np_capacity,
            max_segment=self.max_segment, step_graph=int(self.step_graph), pp_queue=int(self.pp_queue),
            nslab=self.nslab, slab=self.slab,
        )


def config_plain_128() -> Params:
    """128^3 particles, 200 Mpc/h, fine mesh 256^3, int8 coordinates, PP on."""
    return Params(ng=256, nnt=4, nns=4, np_nc=2, izipx=1, box=200.0)


def config_512() -> Params:
    """512^3 particles, 1000 Mpc/h, fine mesh 1024^3, int16 coordinates."""
    return Params(ng=1024, nnt=4, nns=4, np_nc=2, izipx=2, box=1000.0, nic=1)


def config_late_256() -> Params:
    """256^3 particles, 100 Mpc/h, fine mesh 256^3 (np_nc = 4, the reference default),
    int16 coordinates: the clustered-PP configuration, evolved to z ~ 0."""
    return Params(ng=256, nnt=4, nns=4, np_nc=4, izipx=2, box=100.0, nic=1)


def config_small(ng: int = 64, nnt: int = 2, nns: int = 2, np_nc: int = 2, izipx: int = 1,
                 box: float = 100.0) -> Params:
    """Small geometry the oracle finishes in seconds (parity tests)."""
    return Params(ng=ng, nnt=nnt, nns=nns, np_nc=np_nc, izipx=izipx, box=box)
