"""Resistivity (flag_resi 1: resistive_flux and cfl_resi with a fixed eta field) on the
device, through the C ABI, against the oracle.

The FMA-free build agrees with the oracle bit for bit where no exp() enters (uniform or
given eta, no IR); runs with the IR rates and the FMA build are held to the drop-in
tolerance of 1e-10 relative L1 per variable.  The 1D case also checks the resistive decay
rate of a sinusoidal field against the discrete operator's eta*sin(k dx)^2/dx^2.
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import rel_l1
from oracle import oracle as O
from pip_b200 import capi, decomp, ics
from pip_b200.params import PIP_MIXED
from resistive_cases import decay_case, decay_factor

pytestmark = pytest.mark.gpu

TOL = 1e-10


def run_gpu(s, Uh, Um, eta=None, nsteps=0, t_end=0.0):
    with capi.Context(s) as c:
        if eta is not None:
            c.set_resistivity(eta)
        c.upload(Uh, Um)
        c.prologue()
        st, t, n = c.run(nsteps, t_end)
        Uh2, Um2 = c.download()
    return st, t, n, Uh2, Um2


def run_orc(s, Uh, Um, eta=None, nsteps=0, t_end=0.0):
    o = O.Oracle(s, Uh, Um)
    try:
        if eta is not None:
            o.set_resistivity(eta)
        o.prologue()
        st, t, n, _ = o.run(nsteps, t_end)
        Uh2, Um2 = o.state()
    finally:
        o.close()
    return st, t, n, Uh2, Um2


def assert_match(g, o, bitwise):
    assert g[0] == o[0] == 0
    assert g[2] == o[2], "step counts differ: gpu %d, oracle %d" % (g[2], o[2])
    if bitwise:
        assert g[1] == o[1]
        np.testing.assert_array_equal(g[3], o[3])
        np.testing.assert_array_equal(g[4], o[4])
        return
    assert abs(g[1] - o[1]) <= 1e-12 * max(1.0, abs(o[1]))
    err = max(rel_l1(g[3], o[3]).max(), rel_l1(g[4], o[4]).max())
    assert err <= TOL, "relative L1 %.3e > %.1e" % (err, TOL)


def test_resistive_decay_1d(gpu_lib):
    s, Uh, Um = decay_case(128, 1e-2, fp_exact=1)
    g = run_gpu(s, Uh, Um, t_end=1.0)
    o = run_orc(s, Uh, Um, t_end=1.0)
    assert_match(g, o, bitwise=True)
    amp, want = decay_factor(s, g[4], g[1])
    assert abs(amp / want - 1.0) < 1e-5


@pytest.mark.parametrize("exact", [1, 0])
def test_orszag_tang_uniform_eta(gpu_lib, exact):
    s, Uh, Um = ics.orszag_tang(48, flag_resi=1, eta_0=2e-3, fp_exact=exact)
    g = run_gpu(s, Uh, Um, nsteps=15)
    o = run_orc(s, Uh, Um, nsteps=15)
    assert_match(g, o, bitwise=bool(exact))


def test_given_field_and_eta_bound(gpu_lib):
    """A field with a strong spot: cfl_resi bounds dt, and the tile corners' curls enter."""
    s, Uh, Um = ics.orszag_tang(40, flag_resi=1, eta_0=1e-3, fp_exact=1)
    eta = 1e-3 * (1.0 + 30.0 * np.random.default_rng(9).random(Uh.shape[1:]) ** 8)
    g = run_gpu(s, Uh, Um, eta, nsteps=12)
    o = run_orc(s, Uh, Um, eta, nsteps=12)
    assert_match(g, o, bitwise=True)


def test_localised_field_with_walls_and_ir(gpu_lib):
    s, Uh, Um = ics.kelvin_helmholtz(48, 32, flag_resi=11, eta_0=5e-3, fp_exact=1)
    eta = s.eta_field()
    g = run_gpu(s, Uh, Um, eta, nsteps=15)
    o = run_orc(s, Uh, Um, eta, nsteps=15)
    assert_match(g, o, bitwise=False)   # exp() of the IR rates: GPU against libm


def test_with_alpha_c_per_cell(gpu_lib):
    s, Uh, Um = ics.orszag_tang(40, flag_resi=1, eta_0=2e-3, flag_col=5, fp_exact=1)
    g = run_gpu(s, Uh, Um, nsteps=12)
    o = run_orc(s, Uh, Um, nsteps=12)
    assert_match(g, o, bitwise=True)


def test_unit_entry_points(gpu_lib):
    s, Uh, Um = ics.orszag_tang(32, flag_resi=1, eta_0=4e-3, fp_exact=1)
    eta = 4e-3 * (1.0 + np.random.default_rng(1).random(Uh.shape[1:]))
    o = O.Oracle(s, Uh, Um)
    o.set_resistivity(eta)
    with capi.Context(s) as c:
        c.set_resistivity(eta)
        c.upload(Uh, Um)
        dt_g, cm_g = c.cfl()
        dt_o, cm_o = o.cfl()
        o.cmax = cm_o
        assert dt_g == dt_o and cm_g == cm_o
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
    o.close()


def _blocks(s, Uh, Um, world, eta):
    return [decomp.DeviceBlock(decomp.block_of(s, world, r), decomp.scatter(s, Uh, world, r),
                               decomp.scatter(s, Um, world, r),
                               eta=decomp.scatter(s, eta[None], world, r)[0])
            for r in range(world)]


@pytest.mark.parametrize("world", [2, 4])
def test_decomposed_device_loop(gpu_lib, world):
    s, Uh, Um = ics.kelvin_helmholtz(32, 32, flag_resi=11, eta_0=5e-3)
    eta = s.eta_field()
    with capi.Context(s) as c:
        c.set_resistivity(eta)
        c.upload(Uh, Um)
        st1, t1, n1 = c.run(nsteps=8)
        rh, rm = c.download()
    assert st1 == 0 and n1 == 8
    engines = _blocks(s, Uh, Um, world, eta)
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    st = run.run_device(8, check_every=4)
    states = [e.download() for e in engines]
    run.close()
    assert st == 0 and run.steps == 8 and run.time == t1
    assert np.array_equal(decomp.gather(s, [a for a, _ in states]), rh)
    assert np.array_equal(decomp.gather(s, [b for _, b in states]), rm)


def test_rejects(gpu_lib):
    s, Uh, Um = ics.orszag_tang(16, flag_resi=1, eta_0=1e-3)
    p, keep = s.to_params()
    h = ctypes.c_void_p()
    p.precision = PIP_MIXED
    assert capi.lib().pip_ctx_create(ctypes.byref(p), ctypes.byref(h)) == capi.PIP_ERR_PARAM
    p.precision = 0
    p.flag_resi = 2
    assert capi.lib().pip_ctx_create(ctypes.byref(p), ctypes.byref(h)) == capi.PIP_ERR_PARAM
    p.flag_resi = 1
    U = torch.zeros(14 * Uh.shape[1] * Uh.shape[2], dtype=torch.float64, device="cuda")
    assert capi.lib().pip_step_noalloc(ctypes.byref(p), ctypes.c_void_p(U.data_ptr()), 1e-4,
                                       0.0, None) == capi.PIP_ERR_PARAM
    s0, _, _ = ics.orszag_tang(16)
    with capi.Context(s0) as c:
        with pytest.raises(capi.PipError) as e:
            c.set_resistivity(np.zeros(c.shape_h[1:]))
        assert e.value.code == capi.PIP_ERR_PARAM


# ------------------------------------------------------------ anomalous eta (flag_resi 2)

# type 2 with these values switches eta to 11 eta_0 in a cell once its current passes
# j_cri (after ~13 steps on 32^2), after which cfl_resi's bound of the new eta lowers the
# time increment; type 3's drift law is continuous
ANOMALOUS = {"type2": dict(flag_resi=22, eta_0=0.03, j_cri=5.5),
             "type3": dict(flag_resi=32, eta_0=2e-2, vd_cri=150.0)}


@pytest.mark.parametrize("exact", [1, 0])
@pytest.mark.parametrize("law", sorted(ANOMALOUS))
def test_orszag_tang_anomalous_eta(gpu_lib, law, exact):
    """set_resistivity resi_type 2 or 3 at every RK stage (flag_resi 22/32): the eta of each
    stage from its own state, cfl_resi's bound of the last stage's eta in the next dt and in
    the time increment.  A step count and a time limit (the last step is found from the
    lowered time)."""
    s, Uh, Um = ics.orszag_tang(32, fp_exact=exact, **ANOMALOUS[law])
    for kw in (dict(nsteps=30), dict(t_end=0.03)):
        g = run_gpu(s, Uh, Um, **kw)
        o = run_orc(s, Uh, Um, **kw)
        assert_match(g, o, bitwise=bool(exact))


def test_anomalous_eta_1d(gpu_lib):
    s, Uh, Um = decay_case(128, 1e-2, flag_resi=22, j_cri=4e-4, fp_exact=1)
    g = run_gpu(s, Uh, Um, t_end=0.2)
    o = run_orc(s, Uh, Um, t_end=0.2)
    assert_match(g, o, bitwise=True)


def test_anomalous_eta_host_stepped(gpu_lib):
    """The Fortran time loop through the C ABI: cfl, run_solver (pip_step), cfl, then
    dt = min(dt, pip_resi_dt) for cfl_resi's write of the global dt, time += dt."""
    s, Uh, Um = ics.orszag_tang(32, fp_exact=1, **ANOMALOUS["type2"])
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        t = 0.0
        for _ in range(25):
            dt, _ = c.cfl()
            c.run_solver(dt)
            c.cfl()
            t = t + min(dt, c.resi_dt())
        gh, gm = c.download()
    o = run_orc(s, Uh, Um, nsteps=25)
    assert t == o[1]
    np.testing.assert_array_equal(gh, o[3])
    np.testing.assert_array_equal(gm, o[4])


def test_anomalous_eta_refuses_a_decomposition(gpu_lib):
    s, Uh, Um = ics.orszag_tang(32, **ANOMALOUS["type3"])
    with capi.Context(s) as c:
        nb = (ctypes.c_int * 4)(-1, -1, 0, 0)
        assert capi.lib().pip_set_neighbors(c.h, nb) == capi.PIP_ERR_PARAM
