"""Checks of the CPU restatement itself (no GPU): an independent numpy transcription of
the 1D step, conservation, directional symmetry and the reference's analytic Alfven-wave
damping rate (Alfven_Damping.f90:82-97)."""
import math

import numpy as np
import pytest

from numpy_pip1d import Run1D
from oracle import oracle as O
from pip_b200 import ics


@pytest.mark.parametrize("case", ["brio_wu", "exponential", "mirror"])
def test_numpy_restatement_matches_bitwise(case):
    if case == "brio_wu":
        s, Uh, Um = ics.brio_wu(96)
    elif case == "exponential":
        s, Uh, Um = ics.shock_tube_member(80, col=3.0e3, pratio=6.0, dratio=3.0, ion_frac=0.4)
    else:
        s, Uh, Um = ics.brio_wu(64, flag_bnd=[2, 10, 1, 1, 1, 1])
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    r = Run1D(s, Uh, Um)
    r.prologue()
    for _ in range(40):
        dt_o = None
        st, t, n, hist = o.run(nsteps=1, max_hist=1)
        dt_o = hist[0]
        dt_n = r.step()
        assert dt_o == dt_n
    oh, om = o.state()
    np.testing.assert_array_equal(oh[:, 0, :], r.Uh)
    np.testing.assert_array_equal(om[:, 0, :], r.Um)
    o.close()


def test_periodic_conservation():
    """Total mass, momentum and energy of both species are conserved to round-off with
    periodic boundaries (the collision source is antisymmetric, PIP_rot.f90:1366-1367)."""
    s, Uh, Um = ics.orszag_tang(48)
    st, t, n, Uh2, Um2, _ = O.run_case(s, Uh, Um, nsteps=80, threads=4)
    m = 2
    sl = (slice(m, -m), slice(m, -m))
    for k, name in ((0, "mass"), (1, "mx"), (2, "my"), (4, "energy")):
        before = Uh[k][sl].sum() + Um[k][sl].sum()
        after = Uh2[k][sl].sum() + Um2[k][sl].sum()
        scale = np.abs(Uh[k][sl]).sum() + np.abs(Um[k][sl]).sum()
        assert abs(after - before) <= 1e-13 * scale, name


@pytest.mark.parametrize("extra", [
    dict(flag_col=5),
    dict(flag_col=7, flag_resi=1, eta_0=2e-3),
    dict(flag_col=4, flag_ir=3, t_norm=1.5e4, n_norm=1.0e11, t_ir=10.0),
    dict(flag_ir=1, t_norm=1.5e4, n_norm=1.0e11, t_ir=10.0, flag_resi=1, eta_0=1e-3),
])
def test_periodic_conservation_with_extra_physics(extra):
    """The same invariants with alpha_c per cell, resistivity and the set_IR laws: their
    sources are antisymmetric between the species and the resistive terms are fluxes."""
    s, Uh, Um = ics.orszag_tang(40, **extra)
    st, t, n, Uh2, Um2, _ = O.run_case(s, Uh, Um, nsteps=40, threads=4)
    assert st == 0
    m = s.margin[0]
    sl = (slice(m, -m), slice(m, -m))
    for k, name in ((0, "mass"), (1, "mx"), (2, "my"), (4, "energy")):
        before = Uh[k][sl].sum() + Um[k][sl].sum()
        after = Uh2[k][sl].sum() + Um2[k][sl].sum()
        scale = np.abs(Uh[k][sl]).sum() + np.abs(Um[k][sl]).sum()
        assert abs(after - before) <= 1e-13 * scale, name


def test_directional_symmetry():
    """A 1D tube along x equals the same tube along y of a 2D grid with (vx,vy), (bx,by)
    swapped, bit for bit (the reference's debug_direction check, shock_tube.f90:64-123)."""
    s1, Uh1, Um1 = ics.brio_wu(64)
    s2 = s1.overrides(ndim=2, ix0=4, jx0=64, start=(0.0, -0.5, 0.0), end=(4.0, 0.5, 1.0),
                      flag_bnd=[1, 1, 10, 10, 1, 1], flag_divb=0)
    ix, jx, _ = s2.shape
    Uh2 = np.zeros((5, jx, ix))
    Um2 = np.zeros((8, jx, ix))
    perm_h = [0, 2, 1, 3, 4]
    perm_m = [0, 2, 1, 3, 4, 6, 5, 7]
    for k in range(5):
        Uh2[perm_h[k]] = Uh1[k, 0, :][:, None]
    for k in range(8):
        Um2[perm_m[k]] = Um1[k, 0, :][:, None]
    a = O.run_case(s1, Uh1, Um1, nsteps=60)
    b = O.run_case(s2, Uh2, Um2, nsteps=60)
    assert a[2] == b[2] and a[1] == b[1]
    for k in range(5):
        np.testing.assert_array_equal(b[3][perm_h[k]][2:-2, 3], a[3][k, 0, 2:-2])
    for k in range(8):
        np.testing.assert_array_equal(b[4][perm_m[k]][2:-2, 3], a[4][k, 0, 2:-2])


def test_alfven_wave_damping_rate():
    """Strongly coupled two-fluid Alfven wave: energy decays as exp(-2 w_i t) with
    w_i = k^2 B0^2 / (2 col (1-xi)/xi) (Alfven_Damping.f90:86-93)."""
    nx, col, xi, b0, amp = 256, 100.0, 0.5, 1.0, 1e-4
    s, _, _ = ics.brio_wu(nx, start=(0.0, -1.0, -1.0), end=(1.0, 1.0, 1.0), col=col,
                          n_fraction=xi, flag_bnd=[1, 1, 1, 1, 1, 1])
    f_n, f_p, f_p_n, f_p_p = ics.fractions(xi)
    x = s.coordinates()[0][None, :]
    k = 2.0 * math.pi
    wi = 0.5 * k * k * b0 ** 2 / (col * (1.0 - xi) / xi)
    wr = math.sqrt((b0 * k) ** 2 - wi ** 2)
    ro = np.ones_like(x)
    vz = amp * np.cos(k * x)
    bz = -b0 / (b0 ** 2 * k) * amp * (wr * np.cos(k * x) + wi * np.sin(k * x))
    zero = np.zeros_like(x)
    pr = np.full_like(x, 1.0 / s.gm)
    Uh = ics.pv2cq_hd(s, f_n * ro, zero, zero, vz, f_p_n * pr)
    Um = ics.pv2cq_mhd(s, f_p * ro, zero, zero, vz, f_p_p * pr, np.full_like(x, b0), zero, bz)

    def energy(h, m):
        sl = slice(2, -2)
        return float((0.5 * h[3, 0, sl] ** 2 / h[0, 0, sl] + 0.5 * m[3, 0, sl] ** 2 / m[0, 0, sl]
                      + 0.5 * m[7, 0, sl] ** 2).sum())
    t_end = 1.5
    st, t, n, Uh2, Um2, _ = O.run_case(s, Uh, Um, t_end=t_end, threads=4)
    ratio = energy(Uh2, Um2) / energy(Uh, Um)
    measured = -math.log(ratio) / (2.0 * t)
    assert abs(measured - wi) <= 0.1 * wi, (measured, wi)
