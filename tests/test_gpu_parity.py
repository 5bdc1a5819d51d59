"""Parity of the CUDA FP64 path with the CPU restatement, through the C ABI.

Two arithmetic flavours are checked: the FMA-free build (fp_exact=1), which must agree
with the oracle bit for bit wherever no exp() is involved, and the default FMA build,
held to the drop-in tolerance of 1e-10 relative L1 per variable.
"""
import numpy as np
import pytest

from helpers import interior, rel_l1
from oracle import oracle as O
from pip_b200 import capi, ics

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10      # relative L1 per variable, FMA build vs oracle
TOL_EXP = 1e-10       # FMA-free build where exp() (GPU vs libm, <= 1 ulp) enters: drop-in bar


def run_gpu(s, Uh, Um, nsteps=0, t_end=0.0):
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, t, n = c.run(nsteps, t_end)
        Uh2, Um2 = c.download()
    return st, t, n, Uh2, Um2


def run_orc(s, Uh, Um, nsteps=0, t_end=None):
    st, t, n, Uh2, Um2, _ = O.run_case(s, Uh, Um, nsteps=nsteps, t_end=t_end, threads=8)
    return st, t, n, Uh2, Um2


def assert_match(g, o, tol, bitwise=False):
    assert g[0] == o[0] == 0
    assert g[2] == o[2], "step counts differ: gpu %d, oracle %d" % (g[2], o[2])
    if bitwise:
        assert g[1] == o[1]
        np.testing.assert_array_equal(g[3], o[3])
        np.testing.assert_array_equal(g[4], o[4])
        return
    assert abs(g[1] - o[1]) <= 1e-12 * max(1.0, abs(o[1]))
    err = max(rel_l1(g[3], o[3]).max(), rel_l1(g[4], o[4]).max())
    assert err <= tol, "relative L1 %.3e > %.1e" % (err, tol)


@pytest.mark.parametrize("exact", [1, 0])
def test_brio_wu_to_t01(gpu_lib, exact):
    """Config 1: 1D Brio-Wu two-fluid tube, nx=1024, to t=0.1 (about 1900 steps)."""
    s, Uh, Um = ics.brio_wu(1024, fp_exact=exact)
    g = run_gpu(s, Uh, Um, t_end=0.1)
    o = run_orc(s, Uh, Um, t_end=0.1)
    assert_match(g, o, TOL_FP64, bitwise=bool(exact))


@pytest.mark.parametrize("exact", [1, 0])
def test_orszag_tang_64(gpu_lib, exact):
    """Config 2 at 64x64 for 60 steps (periodic, Dedner cleaning)."""
    s, Uh, Um = ics.orszag_tang(64, fp_exact=exact)
    g = run_gpu(s, Uh, Um, nsteps=60)
    o = run_orc(s, Uh, Um, nsteps=60)
    assert_match(g, o, TOL_FP64, bitwise=bool(exact))


_OT1024 = {}


def ot1024_oracle():
    """The oracle's 20 steps of config 2 at its full size, computed once per session."""
    if not _OT1024:
        import os
        s, Uh, Um = ics.orszag_tang(1024)
        st, t, n, oh, om, _ = O.run_case(s, Uh, Um, nsteps=20, threads=os.cpu_count() or 8)
        _OT1024["o"] = (st, t, n, oh, om)
    return _OT1024["o"]


def test_orszag_tang_1024_full_size(gpu_lib):
    """Config 2 on its stated grid, 1024x1024 (+2 ghosts per side), 20 steps, the FMA-free
    build: bit for bit."""
    s, Uh, Um = ics.orszag_tang(1024, fp_exact=1)
    g = run_gpu(s, Uh, Um, nsteps=20)
    assert_match(g, ot1024_oracle(), 0.0, bitwise=True)


# The Dedner potential psi turns rounding differences into ~1e-8 relative differences within
# the first steps of this run (psi is ~1e-4 of |B| and driven by the grid-scale part of
# div B; test_gpu_mixed.py::test_psi_amplifies_white_noise_in_b); the FMA build rounds
# differently from the FMA-free oracle, so its psi is held to this bound and the 13
# physical fields to the drop-in bar.  The FMA-free build above meets the bar on all 14.
TOL_PSI_FMA = 1e-7


def test_orszag_tang_1024_full_size_fma(gpu_lib):
    s, Uh, Um = ics.orszag_tang(1024)
    g = run_gpu(s, Uh, Um, nsteps=20)
    o = ot1024_oracle()
    assert g[0] == o[0] == 0 and g[2] == o[2]
    assert abs(g[1] - o[1]) <= 1e-12 * o[1]
    eh, em = rel_l1(g[3], o[3]), rel_l1(g[4], o[4])
    print("FMA build vs oracle, 13 fields max %.3e, psi %.3e" % (max(eh.max(), em[:8].max()), em[8]))
    assert max(eh.max(), em[:8].max()) <= TOL_FP64
    assert em[8] <= TOL_PSI_FMA


@pytest.mark.parametrize("nx,ny", [(40, 24), (33, 17), (96, 70)])
def test_ragged_tiles(gpu_lib, nx, ny):
    """Interior sizes that are not multiples of the 32x8 tile."""
    s, Uh, Um = ics.orszag_tang(8, ix0=nx, jx0=ny, fp_exact=1)
    g = run_gpu(s, Uh, Um, nsteps=12)
    o = run_orc(s, Uh, Um, nsteps=12)
    assert_match(g, o, 0.0, bitwise=True)


@pytest.mark.parametrize("exact", [1, 0])
@pytest.mark.parametrize("bnd", [[2, 2, 2, 2], [3, 4, 5, 6], [7, 11, 10, 2], [1, 1, 10, 10],
                                 [2, 2, 10, 10], [10, 10, 2, 2]])
def test_boundary_codes(gpu_lib, bnd, exact):
    """Mirror codes with their sign tables, outflow and periodic, incl. corners.  At a mirror
    face the HLL averages of vn and Bn cancel to exactly zero and the L*/R* choice follows
    their sign: the FMA build must round those products alone to stay at the drop-in bar
    (unfused, a mirror wall's tangential fluxes flipped sign at 5% of the state)."""
    s, Uh, Um = ics.orszag_tang(48, flag_bnd=bnd + [1, 1], fp_exact=exact)
    g = run_gpu(s, Uh, Um, nsteps=15)
    o = run_orc(s, Uh, Um, nsteps=15)
    assert_match(g, o, TOL_FP64, bitwise=bool(exact))


def test_no_divb_2d(gpu_lib):
    s, Uh, Um = ics.orszag_tang(40, flag_divb=0, fp_exact=1)
    g = run_gpu(s, Uh, Um, nsteps=20)
    o = run_orc(s, Uh, Um, nsteps=20)
    assert_match(g, o, 0.0, bitwise=True)


@pytest.mark.parametrize("exact", [1, 0])
def test_exponential_collisions(gpu_lib, exact):
    """flag_pip_imp=1 with a stiff alpha_c (the ensemble members' form)."""
    s, Uh, Um = ics.shock_tube_member(300, col=5.0e3, pratio=8.0, dratio=4.0, ion_frac=0.3,
                                      fp_exact=exact)
    g = run_gpu(s, Uh, Um, t_end=0.05)
    o = run_orc(s, Uh, Um, t_end=0.05)
    assert_match(g, o, TOL_EXP if exact else TOL_FP64)


@pytest.mark.parametrize("exact", [1, 0])
def test_ionisation_recombination(gpu_lib, exact):
    """PIP_IR_POWERLAW source on a small Kelvin-Helmholtz layer (reflecting y walls)."""
    s, Uh, Um = ics.kelvin_helmholtz(64, 32, fp_exact=exact)
    g = run_gpu(s, Uh, Um, nsteps=30)
    o = run_orc(s, Uh, Um, nsteps=30)
    assert_match(g, o, TOL_EXP if exact else TOL_FP64)


def test_drop_in_call_sequence(gpu_lib):
    """main.f90's calls one by one (cfl, run_solver, cfl) equal pip_run's fused loop."""
    s, Uh, Um = ics.orszag_tang(32, fp_exact=1)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        t = 0.0
        for _ in range(7):
            dt, _ = c.cfl()
            c.run_solver(dt)
            c.cfl()
            t += dt
        a = c.download()
    g = run_gpu(s, Uh, Um, nsteps=7)
    np.testing.assert_array_equal(a[0], g[3])
    np.testing.assert_array_equal(a[1], g[4])
    assert t == g[1]


def test_unit_entry_points(gpu_lib):
    """pip_cfl, pip_flux, pip_source and pip_fill_ghosts against their oracle routines."""
    s, Uh, Um = ics.orszag_tang(40, fp_exact=1)
    rng = np.random.default_rng(7)
    Uh = Uh * (1 + 1e-3 * rng.standard_normal(Uh.shape))
    Um = Um * (1 + 1e-3 * rng.standard_normal(Um.shape))
    o = O.Oracle(s, Uh, Um)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        # ghost fill
        c.pipbnd()
        o.fill_ghosts()
        gh, gm = c.download()
        oh, om = o.state()
        np.testing.assert_array_equal(gh, oh)
        np.testing.assert_array_equal(gm, om)
        # cfl: dt, cmax and the rewritten state
        dt_g, cm_g = c.cfl()
        dt_o, cm_o = o.cfl()
        o.cmax = cm_o
        assert dt_g == dt_o and cm_g == cm_o
        gh, gm = c.download()
        oh, om = o.state()
        np.testing.assert_array_equal(gh, oh)
        np.testing.assert_array_equal(gm, om)
        # fluxes on faces adjacent to interior cells
        m = s.margin
        ix, jx, _ = s.shape
        for d in (1, 2):
            Fh_g, Fm_g = c.set_flux(d)
            Fh_o, Fm_o = o.flux(d)
            if d == 1:
                sl = (slice(None), slice(m[1], jx - m[1]), slice(m[0] - 1, ix - m[0]))
            else:
                sl = (slice(None), slice(m[1] - 1, jx - m[1]), slice(m[0], ix - m[0]))
            np.testing.assert_array_equal(Fh_g[sl], Fh_o[sl])
            np.testing.assert_array_equal(Fm_g[sl], Fm_o[sl])
        # source (explicit form) and its rewrite of the state
        Sh_g, Sm_g = c.source_pip(1.0e-4)
        Sh_o, Sm_o = o.source(1.0e-4)
        np.testing.assert_array_equal(Sh_g, Sh_o)
        np.testing.assert_array_equal(Sm_g, Sm_o)
        gh, gm = c.download()
        oh, om = o.state()
        np.testing.assert_array_equal(gh, oh)
        np.testing.assert_array_equal(gm, om)
    o.close()


def test_nan_stops_the_loop(gpu_lib):
    """stop_sim: a NaN in the state ends pip_run after the step that carries it."""
    s, Uh, Um = ics.orszag_tang(32)
    Um = Um.copy()
    Um[0, 10, 10] = np.nan
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st, t, n = c.run(nsteps=50)
        assert st == capi.PIP_ERR_NAN
        assert n <= 2
        stop, nan = c.status()
        assert stop == 1 and nan == 1


def test_tiny_dt_stops_the_loop(gpu_lib):
    """stop_sim: dt <= 1e-12 ends the loop with PIP_ERR_DT after that step."""
    s, Uh, Um = ics.brio_wu(64, col=1.0e15)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st, t, n = c.run(nsteps=10)
        assert st == capi.PIP_ERR_DT
        assert n == 1


def test_run_respects_t_end_and_resumes(gpu_lib):
    """Two pip_run calls to t=0.02 then 0.04 equal one call to 0.04 step for step."""
    s, Uh, Um = ics.brio_wu(256, fp_exact=1)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, t1, n1 = c.run(t_end=0.02)
        st, t2, n2 = c.run(t_end=0.04)
        a = c.download()
    o = run_orc(s, Uh, Um, t_end=0.04)
    assert n1 + n2 == o[2]
    assert t2 == o[1]
    np.testing.assert_array_equal(a[0], o[3])
    np.testing.assert_array_equal(a[1], o[4])


def test_newton_reciprocal_within_one_ulp(tmp_path):
    """The FP64 reciprocal of the folded-division solver forms (pip_physics.cuh rcp_: the
    hardware seed and two Newton-Raphson steps) stays within one ulp of the IEEE division
    over 2^22 seeded normal values of every exponent and both signs."""
    import os
    import re
    import subprocess
    from pip_b200 import build as b
    here = os.path.dirname(os.path.abspath(__file__))
    exe = tmp_path / "rcp_check"
    subprocess.run([b.nvcc()] + b.ARCH + ["-O3", "-std=c++17", "--expt-relaxed-constexpr",
                    os.path.join(here, "rcp_check.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    print(out)
    m = re.search(r"values (\d+) max_ulp (\d+) differ (\d+) nonfinite (\d+)", out)
    assert m and int(m.group(1)) == 1 << 22
    assert int(m.group(2)) <= 1 and int(m.group(4)) == 0
