"""alpha_c per cell (flag_col 2..7: set_collisional col_type 1..6) on the device, through
the C ABI, against the oracle.

set_collisional rewrites both energies and recomputes alpha_c at the start of every RK
stage; the second stage's field bounds the next dt (cfl_pn_col).  The FMA-free build
agrees with the oracle bit for bit where alpha_c takes only square roots (col_type 1..4)
and no exp() enters; col_type 5 and 6 raise to the power 0.125 (CUDA pow against libm pow,
<= 2 ulp), so they, the exponential form, the IR rates and the FMA build are held to the
drop-in tolerance of 1e-10 relative L1 per variable.
"""
import ctypes

import numpy as np
import pytest
import torch

from decomp_cases import make_case
from helpers import rel_l1
from oracle import oracle as O
from pip_b200 import capi, decomp, ics
from pip_b200.params import PIP_MIXED

pytestmark = pytest.mark.gpu

TOL = 1e-10


def run_gpu(s, Uh, Um, nsteps=0, t_end=0.0):
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, t, n = c.run(nsteps, t_end)
        Uh2, Um2 = c.download()
        ac = c.alpha_c()
    return st, t, n, Uh2, Um2, ac


def run_orc(s, Uh, Um, nsteps=0, t_end=0.0):
    o = O.Oracle(s, Uh, Um)
    try:
        o.prologue()
        st, t, n, _ = o.run(nsteps, t_end)
        Uh2, Um2 = o.state()
        ac = o.alpha_c()
    finally:
        o.close()
    return st, t, n, Uh2, Um2, ac


def assert_match(g, o, bitwise):
    assert g[0] == o[0] == 0
    assert g[2] == o[2], "step counts differ: gpu %d, oracle %d" % (g[2], o[2])
    if bitwise:
        assert g[1] == o[1]
        for a, b in zip(g[3:], o[3:]):
            np.testing.assert_array_equal(a, b)
        return
    assert abs(g[1] - o[1]) <= 1e-12 * max(1.0, abs(o[1]))
    err = max(rel_l1(g[3], o[3]).max(), rel_l1(g[4], o[4]).max(),
              np.abs(g[5] - o[5]).sum() / np.abs(o[5]).sum())
    assert err <= TOL, "relative L1 %.3e > %.1e" % (err, TOL)


@pytest.mark.parametrize("flag_col", [2, 3, 4, 5, 6, 7])
def test_orszag_tang_each_col_type(gpu_lib, flag_col):
    s, Uh, Um = ics.orszag_tang(48, flag_col=flag_col, fp_exact=1)
    g = run_gpu(s, Uh, Um, nsteps=12)
    o = run_orc(s, Uh, Um, nsteps=12)
    assert_match(g, o, bitwise=flag_col <= 5)
    # the field is the second stage's and varies over the grid
    assert g[5].max() > g[5].min()


@pytest.mark.parametrize("flag_col", [4, 7])
def test_fma_build(gpu_lib, flag_col):
    s, Uh, Um = ics.orszag_tang(48, flag_col=flag_col, fp_exact=0)
    g = run_gpu(s, Uh, Um, nsteps=12)
    o = run_orc(s, Uh, Um, nsteps=12)
    assert_match(g, o, bitwise=False)


@pytest.mark.parametrize("flag_col", [3, 5])
def test_brio_wu_1d(gpu_lib, flag_col):
    s, Uh, Um = ics.brio_wu(256, flag_col=flag_col, fp_exact=1)
    g = run_gpu(s, Uh, Um, t_end=0.01)
    o = run_orc(s, Uh, Um, t_end=0.01)
    assert_match(g, o, bitwise=True)


@pytest.mark.parametrize("flag_col", [5, 6])
def test_exponential_form(gpu_lib, flag_col):
    """flag_pip_imp = 1: the second stage re-derives the first stage's U0 increments with
    the first stage's alpha_c."""
    s, Uh, Um = ics.shock_tube_member(300, col=2.0e3, pratio=8.0, dratio=4.0, ion_frac=0.3,
                                      flag_col=flag_col, fp_exact=1)
    g = run_gpu(s, Uh, Um, nsteps=40)
    o = run_orc(s, Uh, Um, nsteps=40)
    assert_match(g, o, bitwise=False)   # exp() of the exponential form: GPU against libm


def test_ionisation_recombination_and_walls(gpu_lib):
    """PIP_IR_POWERLAW and reflecting y walls (ghost alpha_c = the mirrored cell's)."""
    s, Uh, Um = ics.kelvin_helmholtz(48, 32, flag_col=5, fp_exact=1)
    g = run_gpu(s, Uh, Um, nsteps=15)
    o = run_orc(s, Uh, Um, nsteps=15)
    assert_match(g, o, bitwise=False)   # exp() of the IR rates: GPU against libm


def test_unit_entry_points(gpu_lib):
    """pip_coefficients, pip_get_alpha_c, pip_cfl and pip_source with the field."""
    s, Uh, Um = ics.orszag_tang(40, flag_col=4, fp_exact=1)
    rng = np.random.default_rng(3)
    Uh = Uh.copy()
    Uh[1:4] += 0.2 * Uh[0] * rng.standard_normal(Uh[1:4].shape)
    o = O.Oracle(s, Uh, Um)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.coefficients()
        o.coefficients()
        np.testing.assert_array_equal(c.alpha_c(), o.alpha_c())
        for a, b in zip(c.download(), o.state()):
            np.testing.assert_array_equal(a, b)
        dt_g, cm_g = c.cfl()
        dt_o, cm_o = o.cfl()
        assert dt_g == dt_o and cm_g == cm_o
        Sh_g, Sm_g = c.source_pip(1.0e-4)
        Sh_o, Sm_o = o.source(1.0e-4)
        np.testing.assert_array_equal(Sh_g, Sh_o)
        np.testing.assert_array_equal(Sm_g, Sm_o)
    o.close()


def test_first_call_makes_the_field(gpu_lib):
    """Without pip_coefficients, the first cfl makes the field from the uploaded state
    (the prologue's set_coefficients(U_h,U_m,0))."""
    s, Uh, Um = ics.orszag_tang(32, flag_col=3, fp_exact=1)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        dt_g, _ = c.cfl()
        ag = c.alpha_c()
    o = O.Oracle(s, Uh, Um)
    dt_o, _ = o.cfl()
    ao = o.alpha_c()
    o.close()
    assert dt_g == dt_o
    np.testing.assert_array_equal(ag, ao)


def test_drop_in_call_sequence(gpu_lib):
    """main.f90's calls one by one (cfl, run_solver, cfl) equal pip_run's fused loop."""
    s, Uh, Um = ics.orszag_tang(32, flag_col=4, fp_exact=1)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        t = 0.0
        for _ in range(6):
            dt, _ = c.cfl()
            c.run_solver(dt)
            c.cfl()
            t += dt
        a = c.download()
    g = run_gpu(s, Uh, Um, nsteps=6)
    np.testing.assert_array_equal(a[0], g[3])
    np.testing.assert_array_equal(a[1], g[4])
    assert t == g[1]


def _blocks(s, Uh, Um, world):
    return [decomp.DeviceBlock(decomp.block_of(s, world, r), decomp.scatter(s, Uh, world, r),
                               decomp.scatter(s, Um, world, r)) for r in range(world)]


@pytest.mark.parametrize("case,world", [("ot", 4), ("kh", 4), ("bw", 4)])
def test_decomposed_runs(gpu_lib, case, world):
    """Blocks exchanging halos (host-stepped and device loop) give pip_run's result: the
    exchanged ghost rows' alpha_c is counted on the neighbouring block."""
    s, Uh, Um = make_case(case)
    s = s.overrides(flag_col=5)
    nsteps = 8
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st1, t1, n1 = c.run(nsteps=nsteps)
        rh, rm = c.download()
        ra = c.alpha_c()
    assert st1 == 0 and n1 == nsteps
    engines = _blocks(s, Uh, Um, world)
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    st = run.run_device(nsteps, check_every=4)
    states = [e.download() for e in engines]
    fields = [e.alpha_c()[None] for e in engines]
    run.close()
    assert st == 0 and run.steps == nsteps and run.time == t1
    assert np.array_equal(decomp.gather(s, [a for a, _ in states]), rh)
    assert np.array_equal(decomp.gather(s, [b for _, b in states]), rm)
    # the blocks' fields, ghost layers at the global ends included (on a periodic axis those
    # come from the halo exchange), are the single domain's
    ga = decomp.gather(s, fields)[0]
    bad = np.argwhere(ga != ra)
    assert bad.size == 0, "alpha_c differs at %d cells, e.g. (j, i) %s: %s vs %s" % (
        len(bad), bad[:8].tolist(), ga[tuple(bad[:8].T)], ra[tuple(bad[:8].T)])
    engines = _blocks(s, Uh, Um, world)
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    st = run.run(nsteps)
    dth = list(run.dt_history)
    states = [e.download() for e in engines]
    run.close()
    # the host-stepped blocks (pip_cfl, pip_stage; dt through the host) agree with the fused
    # loop to round-off, as they do with a constant alpha_c
    assert st == 0 and abs(sum(dth) - t1) <= 1e-14 * t1
    hn = decomp.gather(s, [a for a, _ in states])
    mn = decomp.gather(s, [b for _, b in states])
    assert max(rel_l1(hn, rh).max(), rel_l1(mn, rm).max()) <= 1e-11


def test_rejects(gpu_lib):
    s, Uh, Um = ics.orszag_tang(16, flag_col=3)
    p, keep = s.to_params()
    p.precision = PIP_MIXED
    h = ctypes.c_void_p()
    assert capi.lib().pip_ctx_create(ctypes.byref(p), ctypes.byref(h)) == capi.PIP_ERR_PARAM
    p.precision = 0
    # the allocation-free step has no alpha_c field (rejected before the state is touched)
    U = torch.zeros(14 * Uh.shape[1] * Uh.shape[2], dtype=torch.float64, device="cuda")
    assert capi.lib().pip_step_noalloc(ctypes.byref(p), ctypes.c_void_p(U.data_ptr()), 1e-4,
                                       0.0, None) == capi.PIP_ERR_PARAM
