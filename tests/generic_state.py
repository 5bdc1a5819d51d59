"""A generic smooth two-fluid state for derivative tests: every primitive field varies, so
that no minmod triple, wave-speed minimum or |Bn| sits exactly on its kink (the linear-wave
ICs have uniform density, pressure and field, where the discrete map is not
differentiable).  Test infrastructure."""
import numpy as np

from pip_b200 import ics


def generic_fields(s, seed, kmax=3):
    X, Y = ics._grid(s)
    rng = np.random.default_rng(seed)
    Lx = s.end[0] - s.start[0]
    Ly = (s.end[1] - s.start[1]) if s.ndim == 2 else 1.0

    def smooth():
        f = np.zeros_like(X)
        for kx in range(0, kmax + 1):
            for ky in range(0, kmax + 1 if s.ndim == 2 else 1):
                if kx == 0 and ky == 0:
                    continue
                f += rng.normal() * np.cos(2.0 * np.pi * (kx * X / Lx + ky * Y / Ly) + rng.uniform(0, 6.28))
        # a random peak value: no two fields share their extreme values
        return f / np.max(np.abs(f)) * rng.uniform(0.6, 1.0)
    return smooth


def generic_state(s, seed=1, bx=None):
    """(U_h, U_m) of smooth random fields on the grid of s (ghosts included); bx: a uniform
    normal field (1D runs without the Bn jumps that make the HLLD central states
    discontinuous at sm = 0)."""
    f = generic_fields(s, seed)
    ro_i = 0.5 * (1.0 + 0.1 * f())
    ro_n = 0.5 * (1.0 + 0.1 * f())
    vx, vy, vz = 0.05 * f(), 0.05 * f(), 0.03 * f()
    nvx, nvy, nvz = 0.05 * f(), 0.05 * f(), 0.03 * f()
    p_i = 0.4 * (1.0 + 0.1 * f())
    p_n = 0.2 * (1.0 + 0.1 * f())
    bx_f, by, bz = 1.0 + 0.1 * f(), 0.3 + 0.1 * f(), 0.2 * f()
    if bx is not None:
        bx_f = np.full_like(bx_f, bx)
    bx = bx_f
    Uh = ics.pv2cq_hd(s, ro_n, nvx, nvy, nvz, p_n)
    Um = ics.pv2cq_mhd(s, ro_i, vx, vy, vz, p_i, bx, by, bz)
    return Uh, Um
