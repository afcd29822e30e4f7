"""Background expansion, linear power spectrum and host timestep.

The reference reads the expansion table ``s_a_tau_H.txt`` and the IC spectrum
``Pcb_ic.txt`` that ``neutrinos/Pk.py`` makes with CAMB (Pk.py:263-283,
315-321).  CAMB is not available, so this module writes the same table format
from an analytic LCDM(+radiation) background, and gives the Eisenstein & Hu
(1998) no-wiggle spectrum normalised by A_s.  The timestep logic restates
timestep.f90:4-110 with ``expansion``/``dtau_a`` (neutrinos/power_nu.f90:8-54).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

DT0 = 5e-4          # table step in code time (Pk.py:264)
ISTEP_MAX = 100000  # parameters.f90:127
RA_MAX = 0.1        # parameters.f90:128
DT_MAX = 1.0        # variables.f90:27
DT_REFINE = 1.0     # parameters.f90:45
C_KMS = 299792.458


def hubble(a, h0, om, orad, ol):
    """H(a) in km/s/Mpc for flat LCDM with radiation."""
    return 100.0 * h0 * np.sqrt(om / a ** 3 + orad / a ** 4 + ol)


def expansion_table(h0: float, om: float, orad: float, n: int = ISTEP_MAX, a_stop: float = 1.0 / 301):
    """Rows (t, a, tau, H) of s_a_tau_H.txt, built like Pk.py:263-283.

    ``a`` decreases from 1 with t = -i*dt0, a_{i+1} = a_i - omHsq*H(a_i)*a_i^3*dt0;
    entries after the stop keep their initial value (a=1), as Pk.py leaves them.
    tau is conformal time in Mpc/(km/s) units, integrated numerically.
    """
    ol = 1.0 - om - orad
    H0 = 100.0 * h0
    omhsq = 2.0 / 3.0 * math.sqrt(1.0 / om) / H0
    t = -np.arange(n) * DT0
    a = np.ones(n)
    H = np.ones(n) * H0
    i_end = n - 1
    for i in range(n - 1):
        Hai = float(hubble(a[i], h0, om, orad, ol))
        H[i] = Hai
        a[i + 1] = -omhsq * Hai * a[i] ** 3 * DT0 + a[i]
        if a[i + 1] <= a_stop:
            i_end = i + 1
            break
    # conformal time tau(a) = int_0^a da / (a^2 H) in Mpc/(km/s): analytic below the last
    # table entry (radiation + matter), cumulative trapezoid along the table above it
    aa = a[: i_end + 1]
    H0 = 100.0 * h0
    a_last = aa[-1]
    tau_last = 2.0 / (H0 * om) * (math.sqrt(orad + om * a_last) - math.sqrt(orad))
    integ = 1.0 / (aa ** 2 * hubble(aa, h0, om, orad, ol))
    seg = 0.5 * (integ[1:] + integ[:-1]) * (aa[:-1] - aa[1:])
    cum = np.concatenate([[0.0], np.cumsum(seg[::-1])])[::-1]
    tau = np.full(n, 0.0)
    tau[: i_end + 1] = tau_last + cum
    tau[i_end + 1:] = tau[0]
    return np.array([t, a, tau, H], dtype=np.float64)


@dataclasses.dataclass
class Background:
    """Float32 copies of the table, as the reference stores them (variables.f90:10)."""

    stime: np.ndarray
    s2a: np.ndarray
    s2tau: np.ndarray
    s2H: np.ndarray
    ia: int = 1  # 1-based cursor (variables.f90:11)

    @classmethod
    def from_table(cls, tab: np.ndarray) -> "Background":
        f = tab.astype(np.float32)
        return cls(f[0].copy(), f[1].copy(), f[2].copy(), f[3].copy())

    def _s(self, arr, i):  # 1-based access
        return float(arr[i - 1])

    def init_cursor(self, a: float) -> None:
        """initialize.f90:93-96."""
        ia = 1
        while self._s(self.s2a, ia + 1) >= a and ia < ISTEP_MAX:
            ia += 1
        self.ia = ia

    def expansion(self, a: float, dt0: float) -> float:
        """power_nu.f90:8-35 (FP64 internals on FP32 table entries, FP32 result)."""
        a8 = float(np.float64(np.float32(a)))
        i1 = self.ia
        while self._s(self.s2a, i1) <= a8 and i1 > 1:
            i1 -= 1
        self.ia = i1
        tdoa = (self._s(self.stime, i1 + 1) - self._s(self.stime, i1)) / (self._s(self.s2a, i1 + 1) - self._s(self.s2a, i1))
        t_x = self._s(self.stime, i1) + tdoa * (a8 - self._s(self.s2a, i1)) + float(np.float32(dt0))
        i2 = i1
        while self._s(self.stime, i2 + 1) < t_x and i2 > 1:
            i2 -= 1
        adot = (self._s(self.s2a, i2 + 1) - self._s(self.s2a, i2)) / (self._s(self.stime, i2 + 1) - self._s(self.stime, i2))
        a_x = self._s(self.s2a, i2) + adot * (t_x - self._s(self.stime, i2))
        return float(np.float32(a_x - a8))

    def dtau_a(self, a: float, tau: float, da0: float) -> float:
        """power_nu.f90:37-54 (FP32)."""
        f = np.float32
        a0 = f(a) + f(da0)
        i1 = self.ia - 1
        while self._s(self.s2a, i1) <= a0 and i1 > 1:
            i1 -= 1
        i2 = i1 + 1
        tdoa = f((f(self._s(self.stime, i2)) - f(self._s(self.stime, i1))) / (f(self._s(self.s2a, i2)) - f(self._s(self.s2a, i1))))
        t_x = f(f(self._s(self.stime, i1)) + tdoa * (a0 - f(self._s(self.s2a, i1))))
        taudot = f((f(self._s(self.s2tau, i2)) - f(self._s(self.s2tau, i1))) / (f(self._s(self.stime, i2)) - f(self._s(self.stime, i1))))
        return float(f(f(self._s(self.s2tau, i1)) + taudot * (t_x - f(self._s(self.stime, i1))) - f(tau)))


@dataclasses.dataclass
class StepState:
    """The scalars of ``sim`` and ``variables`` that the timestep reads and writes."""

    a: float
    t: float = 0.0
    tau: float = 0.0
    timestep: int = 0
    dt: float = 0.0
    dt_old: float = 0.0
    dt_pm1: float = 1e3
    dt_pm2: float = 1e3
    dt_pm3: float = 1e3
    dt_pp: float = 1e3
    dt_vmax: float = 1e3
    vz_max: float = 0.0
    a_mid: float = 0.0
    cur_checkpoint: int = 2  # next target; main.f90:19 steps past the checkpoint it resumed from
    checkpoint_step: bool = False
    final_step: bool = False


def timestep(bg: Background, st: StepState, z_checkpoint: list[float]) -> None:
    """timestep.f90:4-110 for one image; z_checkpoint is 1-based via cur_checkpoint."""
    f = np.float32
    st.dt_old = st.dt
    st.timestep += 1
    dt_e = f(DT_MAX)
    ntry = 0
    while True:
        ntry += 1
        da = f(bg.expansion(st.a, dt_e))
        ra = f(da / (f(st.a) + da))
        if ra > f(RA_MAX):
            dt_e = f(dt_e * (f(RA_MAX) / ra))
        else:
            break
        if ntry > 10:
            break
    dt = f(min(dt_e, f(st.dt_pm1), f(st.dt_pm2), f(st.dt_pm3), f(DT_REFINE) * f(st.dt_pp), f(st.dt_vmax)))
    da = f(bg.expansion(st.a, dt))
    st.checkpoint_step = False
    n_checkpoint = len(z_checkpoint)
    z_next = f(z_checkpoint[st.cur_checkpoint - 1])
    a_next = f(1.0) / (f(1) + z_next)
    if da >= a_next - f(st.a):
        st.checkpoint_step = True
        if st.cur_checkpoint == n_checkpoint:
            st.final_step = True
        it = 0
        while (abs((f(st.a) + da) / a_next - f(1)) >= f(1e-6) or (f(st.a) + da) > 1) and it < 100:
            dt = f(dt * (a_next - f(st.a)) / da)
            da = f(bg.expansion(st.a, dt))
            it += 1
    st.a_mid = float(f(st.a) + (da / f(2)))
    dtau = bg.dtau_a(st.a, st.tau, da)
    st.tau = float(f(st.tau) + f(dtau))
    st.t = float(f(st.t) + dt)
    st.a = float(f(st.a) + da)
    st.dt = float(dt)


# ---------------------------------------------------------------------------------
# Linear spectrum: Eisenstein & Hu (1998) no-wiggle transfer function, A_s-normalised.
# ---------------------------------------------------------------------------------
def eh_nowiggle_T(k_hmpc, h, om, ob, tcmb=2.7255):
    """EH98 eqs. 26-31; k in h/Mpc."""
    k = np.asarray(k_hmpc, dtype=np.float64)
    theta = tcmb / 2.7
    omh2 = om * h * h
    obh2 = ob * h * h
    fb = ob / om
    s = 44.5 * np.log(9.83 / omh2) / np.sqrt(1.0 + 10.0 * obh2 ** 0.75)  # Mpc
    alpha_g = 1.0 - 0.328 * np.log(431.0 * omh2) * fb + 0.38 * np.log(22.3 * omh2) * fb * fb
    kmpc = k * h
    gamma_eff = om * h * (alpha_g + (1.0 - alpha_g) / (1.0 + (0.43 * kmpc * s) ** 4))
    q = k * theta * theta / gamma_eff
    L0 = np.log(2.0 * math.e + 1.8 * q)
    C0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
    return L0 / (L0 + C0 * q * q)


def growth_cpt(a, om, ol):
    """Carroll-Press-Turner growth, Dgrow of main.f90:66-79 without the a=1 normalisation:
    equals a in matter domination."""
    hsq = om / a ** 3 + (1 - om - ol) / a ** 2 + ol
    oma = om / (a ** 3 * hsq)
    ola = ol / hsq
    ga = 2.5 * oma / (oma ** (4.0 / 7) - ola + (1 + oma / 2) * (1 + ola / 70))
    return a * ga


def linear_power(k_hmpc, a, p) -> np.ndarray:
    """P(k,a) in (Mpc/h)^3 for the Params cosmology (A_s, n_s at k_pivot=0.05/Mpc)."""
    k = np.asarray(k_hmpc, dtype=np.float64)
    h = p.h0
    om = p.omega_m
    T = eh_nowiggle_T(k, h, om, p.omega_b)
    kpiv = 0.05 / h  # parameters.f90:125 (k_o in h/Mpc)
    H0c = 100.0 / C_KMS  # H0/c in h/Mpc
    D = growth_cpt(a, om, p.omega_l)
    with np.errstate(divide="ignore", invalid="ignore"):
        d2 = (4.0 / 25.0) * (k / H0c) ** 4 * T ** 2 * (D / om) ** 2 * p.A_s * (k / kpiv) ** (p.n_s - 1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(k > 0, 2.0 * math.pi ** 2 * d2 / np.where(k > 0, k, 1.0) ** 3, 0.0)
    return P


def vfactor(a, om, ol) -> float:
    """ic.f90:937-945."""
    lm = ol / om
    km = (1 - om - ol) / om
    H = 2 / (3 * math.sqrt(a ** 3)) * math.sqrt(1 + a * km + a ** 3 * lm)
    return a ** 2 * H


def fixed_steps(bg: Background, a_start: float, a_end: float, nsteps: int):
    """A fixed-step schedule: `nsteps` KDK steps of equal code time dt from a_start to
    a_end, for runs quoted at a fixed step count (the reference's own timestep is
    adaptive, timestep.f90:4-110).  Returns [(dt, dt_old, a_mid, a_next)] per step, with
    a_mid = a + da/2 and da from the same table interpolation (power_nu.f90:8-35); the
    closing half drift is (dt_old=0, dt=dt) as main.f90:39-41 does at a checkpoint."""
    if nsteps < 1 or not (0 < a_start < a_end <= 1):
        raise ValueError("need nsteps >= 1 and 0 < a_start < a_end <= 1")
    f = np.float32
    bg.init_cursor(a_start)
    target = float(f(a_end) - f(a_start))
    lo, hi = 0.0, 1.0
    while float(bg.expansion(a_start, hi)) < target:
        hi *= 2
        if hi > 1e6:
            raise ValueError("a_end not reached by the expansion table")
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        bg.init_cursor(a_start)
        if float(bg.expansion(a_start, mid)) < target:
            lo = mid
        else:
            hi = mid
    dt = float(f(0.5 * (lo + hi) / nsteps))
    out = []
    a = float(f(a_start))
    bg.init_cursor(a)
    dt_old = 0.0
    for _ in range(nsteps):
        da = f(bg.expansion(a, dt))
        a_mid = float(f(a) + da / f(2))
        a_next = float(f(a) + da)
        out.append((dt, dt_old, a_mid, a_next))
        dt_old = dt
        a = a_next
    return out
