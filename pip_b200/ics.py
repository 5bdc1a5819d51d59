"""Initial conditions of the benchmark configurations, as PIP's IC routines build them.

Every IC returns ``(settings, U_h, U_m)``: the settings of the run and the conserved
arrays in the Fortran layout ``U(ix,jx,kx,nvar)``, i.e. numpy arrays of shape
``(nvar, jx, ix)`` (kx = 1) in C order.  Primitive fields are converted with ``pv2cq_hd``
and ``pv2cq_mhd`` (Scheme_rot.f90:30-79, flag_b_stg = 0), keeping the Fortran operation
order.  The two-fluid split follows the reference's convention (``shock_tube.f90:28-37``,
``Orszag_Tang.f90:23-33``): densities rho_n = f_n rho, rho_i = f_p rho; pressures
p_n = f_n/(f_n+2 f_p) p and p_i = 2 f_p/(f_n+2 f_p) p (electrons double the ion pressure).
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

from .params import PIP_IR_POWERLAW, Settings

PI = 3.1415926535897932  # parameters.f90 pi


def fractions(n_fraction: float):
    """f_n, f_p, f_p_n, f_p_p of the IC routines (shock_tube.f90:28-37)."""
    f_n = n_fraction
    f_p = 1.0 - n_fraction
    f_p_n = f_n / (f_n + 2.0 * f_p)
    f_p_p = 2.0 * f_p / (f_n + 2.0 * f_p)
    return f_n, f_p, f_p_n, f_p_p


def pv2cq_hd(s: Settings, de, vx, vy, vz, pr) -> np.ndarray:
    """pv2cq_hd, Scheme_rot.f90:30-40."""
    gm = s.gm
    U = np.zeros((5,) + de.shape)
    U[0] = de
    U[1] = de * vx
    U[2] = de * vy
    U[3] = de * vz
    U[4] = pr / (gm - 1.0) + 0.5 * de * (vx * vx + vy * vy + vz * vz)
    return U


def pv2cq_mhd(s: Settings, de, vx, vy, vz, pr, bx, by, bz) -> np.ndarray:
    """pv2cq_mhd, Scheme_rot.f90:43-79 (cell-centred B); psi starts at zero."""
    gm = s.gm
    U = np.zeros((s.nvar_m,) + de.shape)
    U[0] = de
    U[1] = de * vx
    U[2] = de * vy
    U[3] = de * vz
    U[4] = (pr / (gm - 1.0) + 0.5 * de * (vx * vx + vy * vy + vz * vz)
            + 0.5 * (bx * bx + by * by + bz * bz))
    U[5] = bx
    U[6] = by
    U[7] = bz
    return U


def _grid(s: Settings):
    x, y, _, _, _, _ = s.coordinates()
    ix, jx, _ = s.shape
    X = np.broadcast_to(x[None, :], (jx, ix)).copy()
    Y = np.broadcast_to(y[:, None], (jx, ix)).copy()
    return X, Y


def brio_wu(nx: int = 1024, **kw) -> Tuple[Settings, np.ndarray, np.ndarray]:
    """1D two-fluid Brio-Wu shock tube: rho 1 / 0.125, p 1 / 0.1, Bx 0.75, By +1 / -1,
    v = 0, x in [-0.5, 0.5], outflow (flag_bnd 10) both sides, 50 % neutral by mass,
    alpha_c = 100, gamma 5/3, CFL 0.3, to t = 0.1.  The states are the Brio-Wu values of
    shock_tube.f90:129-130 with a sharp jump at x = 0."""
    s = Settings(ndim=1, ix0=nx, start=(-0.5, -1.0, -1.0), end=(0.5, 1.0, 1.0),
                 flag_bnd=[10, 10, 10, 10, 10, 10], n_fraction=0.5, col=100.0,
                 safety=0.3, tend=0.1, flag_divb=0)
    s = s.overrides(**kw)
    f_n, f_p, f_p_n, f_p_p = fractions(s.n_fraction)
    X, _ = _grid(s)
    left = X < 0.0
    ro = np.where(left, 1.0, 0.125)
    pr = np.where(left, 1.0, 0.1)
    by = np.where(left, 1.0, -1.0)
    zero = np.zeros_like(X)
    bx = np.full_like(X, 0.75)
    U_h = pv2cq_hd(s, f_n * ro, zero, zero, zero, f_p_n * pr)
    U_m = pv2cq_mhd(s, f_p * ro, zero, zero, zero, f_p_p * pr, bx, by, zero)
    return s, U_h, U_m


def orszag_tang(n: int = 1024, **kw) -> Tuple[Settings, np.ndarray, np.ndarray]:
    """2D two-fluid Orszag-Tang vortex on [0,1]^2, periodic (Orszag_Tang.f90:1-95):
    rho = 25/(36 pi), p = 5/(12 pi), v = (-sin 2 pi y, sin 2 pi x),
    B = (-sin 2 pi y, sin 4 pi x)/sqrt(4 pi); 90 % neutral by mass, alpha_c = 1e3,
    Dedner cleaning on (flag_divb = 1, the reference default), CFL 0.3."""
    s = Settings(ndim=2, ix0=n, jx0=n, start=(0.0, 0.0, 0.0), end=(1.0, 1.0, 1.0),
                 flag_bnd=[1, 1, 1, 1, 1, 1], n_fraction=0.9, col=1.0e3, safety=0.3,
                 flag_divb=1, db_clean=0.7)
    s = s.overrides(**kw)
    f_n, f_p, f_p_n, f_p_p = fractions(s.n_fraction)
    X, Y = _grid(s)
    v0 = 1.0
    b0 = 1.0 / math.sqrt(4.0 * PI)
    ro_h = np.full_like(X, 25.0 / (36.0 * PI) * f_n)
    ro_m = np.full_like(X, 25.0 / (36.0 * PI) * f_p)
    p_h = np.full_like(X, 5.0 / (12.0 * PI) * f_p_n)
    p_m = np.full_like(X, 5.0 / (12.0 * PI) * f_p_p)
    vx = v0 * (-np.sin(2.0 * PI * Y))
    vy = v0 * np.sin(2.0 * PI * X)
    bx = b0 * (-np.sin(2.0 * PI * Y))
    by = b0 * np.sin(4.0 * PI * X)
    zero = np.zeros_like(X)
    U_h = pv2cq_hd(s, ro_h, vx, vy, zero, p_h)
    U_m = pv2cq_mhd(s, ro_m, vx, vy, zero, p_m, bx, by, zero)
    return s, U_h, U_m


def kelvin_helmholtz(nx: int = 2048, ny: int = 1024, seed: int = 1234, **kw):
    """2D partially ionised Kelvin-Helmholtz layer: periodic in x, reflecting (flag_bnd 2)
    in y, vx = 0.5 tanh(y/0.05), rho = 1, p = 1/gamma, Bx = 0.1, seeded
    vy ~ U[-1e-3, 1e-3] exp(-(y/0.1)^2), x in [-1, 1], y in [-0.5, 0.5]; 50 % neutral by
    mass; ionisation/recombination by PIP_IR_POWERLAW with chi = 5, the coefficients
    chosen so that the initial state is in ionisation balance.  The shape follows
    KH.f90:1-145; the IR law and the conduction are new."""
    s = Settings(ndim=2, ix0=nx, jx0=ny, start=(-1.0, -0.5, 0.0), end=(1.0, 0.5, 1.0),
                 flag_bnd=[1, 1, 2, 2, 1, 1], n_fraction=0.5, col=100.0, safety=0.3,
                 flag_divb=0, flag_ir=PIP_IR_POWERLAW, flag_ir_type=1, ir_chi=5.0)
    s = s.overrides(**kw)
    f_n, f_p, f_p_n, f_p_p = fractions(s.n_fraction)
    X, Y = _grid(s)
    gm = s.gm
    ro = np.ones_like(X)
    pr = np.full_like(X, 1.0 / gm)
    vx = 0.5 * np.tanh(Y / 0.05)
    rng = np.random.default_rng(seed)
    vy = rng.uniform(-1.0e-3, 1.0e-3, size=X.shape) * np.exp(-(Y / 0.1) ** 2)
    zero = np.zeros_like(X)
    bx = np.full_like(X, 0.1)
    if s.flag_ir == PIP_IR_POWERLAW and s.ir_ion_coef == 0.0 and s.ir_rec_coef == 0.0:
        # ionisation balance Gm_rec rho_i = Gm_ion rho_n at the initial temperature
        te = 0.5 * gm * (f_p_p / f_p) * (1.0 / gm)
        rec = 1.0
        ion = rec * (f_p / f_n) * math.exp(s.ir_chi / te)
        s = s.overrides(ir_rec_coef=rec, ir_ion_coef=ion)
    U_h = pv2cq_hd(s, f_n * ro, vx, vy, zero, f_p_n * pr)
    U_m = pv2cq_mhd(s, f_p * ro, vx, vy, zero, f_p_p * pr, bx, zero, zero)
    return s, U_h, U_m


def wave_damping(nx: int = 512, ny: int = 256, seed: int = 5150, amp: float = 1.0e-4,
                 kmax: int = 8, **kw):
    """2D two-fluid linear wave damping on [0,1]x[0,0.5], periodic: rho = 1 (50 % ions),
    p = 0.6, B0 = 1 along x, alpha_c = 10, plus a seeded velocity perturbation of
    amplitude ``amp`` built from random Fourier modes with |k| <= kmax, given to both
    species (linear_wave.f90 / Alfven_Damping.f90 shape)."""
    s = Settings(ndim=2, ix0=nx, jx0=ny, start=(0.0, 0.0, 0.0), end=(1.0, 0.5, 1.0),
                 flag_bnd=[1, 1, 1, 1, 1, 1], n_fraction=0.5, col=10.0, safety=0.3,
                 flag_divb=0)
    s = s.overrides(**kw)
    f_n, f_p, f_p_n, f_p_p = fractions(s.n_fraction)
    X, Y = _grid(s)
    dv = velocity_modes(X, Y, (s.end[0] - s.start[0]), (s.end[1] - s.start[1]), seed, amp, kmax)
    zero = np.zeros_like(X)
    ro = np.ones_like(X)
    pr = np.full_like(X, 0.6)
    bx = np.ones_like(X)
    U_h = pv2cq_hd(s, f_n * ro, dv[0], dv[1], zero, f_p_n * pr)
    U_m = pv2cq_mhd(s, f_p * ro, dv[0], dv[1], zero, f_p_p * pr, bx, zero, zero)
    return s, U_h, U_m


def velocity_modes(X, Y, Lx, Ly, seed, amp, kmax):
    """Sum of random Fourier modes (integer wave numbers, 0 < |k| <= kmax) scaled to a
    maximum amplitude ``amp`` for each velocity component."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(2):
        f = np.zeros_like(X)
        for kx in range(-kmax, kmax + 1):
            for ky in range(0, kmax + 1):
                if (kx == 0 and ky == 0) or kx * kx + ky * ky > kmax * kmax:
                    continue
                if ky == 0 and kx < 0:
                    continue
                a, ph = rng.normal(), rng.uniform(0.0, 2.0 * PI)
                f += a * np.cos(2.0 * PI * (kx * X / Lx + ky * Y / Ly) + ph)
        f *= amp / np.max(np.abs(f))
        out.append(f)
    return out


def lte_nexcite(s: Settings, ro_h: np.ndarray, ro_m: np.ndarray, pr_m: np.ndarray) -> np.ndarray:
    """Nexcite (6, ...) for set_IR type 4 in local thermodynamic equilibrium: levels 1-5 share
    rho_n in the Saha-Boltzmann ratios n_k/n_i = n_e g_k/(2 g_i) (2 pi m_e k T/h^2)^(-3/2)
    exp(chi_k/kT) at the electron temperature and density set_IR type 4 uses
    (Te_p*T_norm/tfac, rho_i*n_norm/n0fac; PIP_rot.f90:240-258), the form KHnlev.f90:74-93
    sets its populations with; level 6 is rho_i."""
    gm = s.gm
    if s.flag_col % 2 == 1:
        tfac = s.t_norm / (float(np.float32(5.0) / np.float32(3.0)) * s.f_p_p_ini / s.f_p_ini)
    else:
        tfac = s.beta / 2.0 * s.f_p_p_ini * 5.0 / 6.0 / s.f_p_ini
    te = 0.5 * gm * (pr_m / ro_m) * s.t_norm / tfac
    ne = ro_m * s.n_norm / s.n0fac
    kb, me, h = 1.38064852e-23, 9.10938356e-31, 6.62607004e-34
    chi = np.array([13.6, 3.4, 1.51, 0.85, 0.54]) * 1.602176634e-19
    g = np.array([2.0, 8.0, 18.0, 32.0, 50.0])
    saha = (2.0 * PI * me * kb * te / (h * h)) ** -1.5
    ratio = np.stack([ne * g[k] / 2.0 * saha * np.exp(chi[k] / (kb * te)) for k in range(5)])
    lev = ratio / ratio.sum(axis=0) * ro_h
    return np.concatenate([lev, ro_m[None]], axis=0)


def _fpp_for(s: Settings, te_p0: float) -> float:
    """f_p_p_ini (with f_p_ini = 1) that makes set_IR type 4's electron temperature
    Te_p*T_norm/tfac equal T_norm where Te_p = te_p0 (tfac of PIP_rot.f90:240-248)."""
    if s.flag_col % 2 == 1:
        return s.t_norm / te_p0 / float(np.float32(5.0) / np.float32(3.0))
    return te_p0 * 2.0 / s.beta * 6.0 / 5.0


def nlevel_tube(nx: int = 512, **kw):
    """1D two-fluid shock tube with set_IR type 4 (the 6-level hydrogen model): the Brio-Wu
    states of brio_wu() (rho 1 / 0.125, p 1 / 0.1, Bx 0.75, By +1 / -1, 50 % neutral by mass),
    T_norm 6500 K, n_norm 1e17 m^-3, tfac such that the left ion state's electron
    temperature is T_norm, populations in LTE (lte_nexcite), outflow boundaries.  Returns
    (settings, U_h, U_m, Nexcite)."""
    s = Settings(ndim=1, ix0=nx, start=(-0.5, -1.0, -1.0), end=(0.5, 1.0, 1.0),
                 flag_bnd=[10, 10, 10, 10, 10, 10], n_fraction=0.5, col=100.0, safety=0.3,
                 tend=0.1, flag_divb=0, flag_ir=4, flag_ir_type=1, t_norm=6500.0,
                 n_norm=1.0e17, t_ir=1.0e-3)
    s = s.overrides(**kw)
    f_n, f_p, f_p_n, f_p_p = fractions(s.n_fraction)
    if "f_p_p_ini" not in kw:
        s = s.overrides(f_p_ini=1.0, f_p_p_ini=_fpp_for(s, 0.5 * s.gm * f_p_p / f_p))
    X, _ = _grid(s)
    left = X < 0.0
    ro = np.where(left, 1.0, 0.125)
    pr = np.where(left, 1.0, 0.1)
    by = np.where(left, 1.0, -1.0)
    zero = np.zeros_like(X)
    bx = np.full_like(X, 0.75)
    U_h = pv2cq_hd(s, f_n * ro, zero, zero, zero, f_p_n * pr)
    U_m = pv2cq_mhd(s, f_p * ro, zero, zero, zero, f_p_p * pr, bx, by, zero)
    nex = lte_nexcite(s, f_n * ro, f_p * ro, f_p_p * pr)
    return s, U_h, U_m, nex


def nlevel_orszag_tang(n: int = 128, **kw):
    """The two-fluid Orszag-Tang vortex of orszag_tang() with set_IR type 4: T_norm 6500 K,
    n_norm 1e17 m^-3, tfac such that the uniform initial ion state's electron temperature is
    T_norm, LTE populations.  Returns (settings, U_h, U_m, Nexcite)."""
    s0, U_h, U_m = orszag_tang(n, **{k: v for k, v in kw.items()
                                     if k not in ("flag_ir", "flag_ir_type", "t_norm", "n_norm",
                                                  "t_ir", "nlev_deriv", "n0fac", "f_p_ini",
                                                  "f_p_p_ini")})
    ro_m, pr_m = U_m[0], None
    f_n, f_p, f_p_n, f_p_p = fractions(s0.n_fraction)
    pm0 = 5.0 / (12.0 * PI) * f_p_p
    rm0 = 25.0 / (36.0 * PI) * f_p
    te_p0 = 0.5 * s0.gm * pm0 / rm0
    s = s0.overrides(flag_ir=4, flag_ir_type=1, t_norm=6500.0, n_norm=1.0e17, t_ir=1.0e-3)
    s = s.overrides(**kw)
    if "f_p_p_ini" not in kw:
        s = s.overrides(f_p_ini=1.0, f_p_p_ini=_fpp_for(s, te_p0))
    pr_m = np.full_like(ro_m, pm0)
    nex = lte_nexcite(s, U_h[0], ro_m, pr_m)
    return s, U_h, U_m, nex


def ensemble_members(n_runs: int = 512, seed: int = 4242):
    """Parameters of the batched ensemble of 1D shock tubes: nx log-uniform in
    [256, 8192], alpha_c log-uniform in [1e-1, 1e4], pressure ratio U[2, 20], density
    ratio U[2, 10], ion mass fraction U[0.05, 0.95]."""
    rng = np.random.default_rng(seed)
    nx = np.exp(rng.uniform(math.log(256), math.log(8192), n_runs)).round().astype(int)
    col = np.exp(rng.uniform(math.log(0.1), math.log(1.0e4), n_runs))
    pratio = rng.uniform(2.0, 20.0, n_runs)
    dratio = rng.uniform(2.0, 10.0, n_runs)
    ion_frac = rng.uniform(0.05, 0.95, n_runs)
    return [dict(nx=int(nx[r]), col=float(col[r]), pratio=float(pratio[r]),
                 dratio=float(dratio[r]), ion_frac=float(ion_frac[r])) for r in range(n_runs)]


def shock_tube_member(nx: int, col: float, pratio: float, dratio: float, ion_frac: float, **kw):
    """One ensemble member: Brio-Wu-like tube with left/right ratios (left state rho = 1,
    p = 1), Bx = 0.75, By = +1/-1, ion mass fraction ``ion_frac``, exponential collision
    form (flag_pip_imp = 1) because alpha_c reaches 1e4."""
    s, _, _ = brio_wu(nx, col=col, n_fraction=1.0 - ion_frac, flag_pip_imp=1, **kw)
    f_n, f_p, f_p_n, f_p_p = fractions(s.n_fraction)
    X, _ = _grid(s)
    left = X < 0.0
    ro = np.where(left, 1.0, 1.0 / dratio)
    pr = np.where(left, 1.0, 1.0 / pratio)
    by = np.where(left, 1.0, -1.0)
    zero = np.zeros_like(X)
    bx = np.full_like(X, 0.75)
    U_h = pv2cq_hd(s, f_n * ro, zero, zero, zero, f_p_n * pr)
    U_m = pv2cq_mhd(s, f_p * ro, zero, zero, zero, f_p_p * pr, bx, by, zero)
    return s, U_h, U_m
