"""Implicit anisotropic conduction of the ions (HC(U_m,nvar_m,1) with the 9-point matrix
and BiCGstab, include/pip_gpu.h pip_conduction) against the oracle, alone and inside whole
runs with ionisation/recombination, plus the FP32-inner / FP64-refinement form."""
import numpy as np
import pytest

from generic_state import generic_state
from helpers import interior, rel_l1
from oracle import oracle as O
from pip_b200 import capi, ics
from pip_b200.params import PIP_FP64, PIP_MIXED

pytestmark = pytest.mark.gpu


def kh_case(nx=48, ny=24, kapper=1.0, tol=1.0e-12, seed=3, **kw):
    s, _, _ = ics.kelvin_helmholtz(nx, ny, flag_heat=1, kapper=kapper, hc_error=tol,
                                   hc_max=2000, **kw)
    Uh, Um = generic_state(s, seed)
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    Uh0, Um0 = o.state()
    return s, o, Uh0, Um0


@pytest.mark.parametrize("kapper", [0.1, 1.0, 10.0])
def test_conduction_matches_oracle(gpu_lib, kapper):
    s, o, Uh0, Um0 = kh_case(kapper=kapper)
    dt, _ = o.cfl()
    h0, m0 = o.state()
    st_o, it_o, rr_o = o.conduction(dt)
    o.fill_ghosts()
    oh, om = o.state()
    o.close()
    with capi.Context(s) as c:
        c.upload(h0, m0)
        st, it, rr = c.conduction(dt)
        c.pipbnd()
        gh, gm = c.download()
    assert st_o == 0 and st == 0 and rr <= 1e-12
    # BiCGstab's iteration count depends on rounding (the GPU sums the dot products in
    # another order and forms the matrix entries from face factors).  Up to tens of
    # iterations the count follows the oracle's; at kapper = 10 (about 200 iterations to
    # 1e-12) the residual history is erratic and GPU summation orders have given 209 to 330
    # against the oracle's 211, so there only convergence and the solution are compared.
    print("kapper", kapper, "iterations gpu", it, "oracle", it_o)
    if kapper <= 1.0:
        assert abs(it - it_o) <= max(3, 0.1 * it_o), (it, it_o)
    else:
        assert it <= 2000
    assert rel_l1(interior(gm, s), interior(om, s)).max() <= 1e-10
    assert np.array_equal(interior(gh, s), interior(oh, s))


@pytest.mark.parametrize("bnd", [[1, 1, 2, 2, 1, 1], [10, 10, 10, 10, 1, 1]])
def test_run_with_conduction_and_ir_matches_oracle(gpu_lib, bnd):
    s, o, Uh0, Um0 = kh_case(kapper=1.0, flag_bnd=bnd)
    st_o, t_o, n_o, hist = o.run(nsteps=15, max_hist=15)
    oh, om = o.state()
    o.close()
    with capi.Context(s) as c:
        c.upload(Uh0, Um0)
        st, t, n = c.run(nsteps=15)
        gh, gm = c.download()
        iters = c.conduction_iterations
    assert st_o == 0 and st == 0 and n == 15 and iters > 0
    assert abs(t - t_o) <= 1e-12 * t_o
    assert max(rel_l1(interior(gh, s), interior(oh, s)).max(),
               rel_l1(interior(gm, s), interior(om, s)).max()) <= 1e-10


def test_mixed_refinement_reaches_fp64_residual(gpu_lib):
    """FP32 BiCGstab on the correction, FP64 residual and update: same solution as the FP64
    solve within the residual target."""
    s, o, Uh0, Um0 = kh_case(kapper=3.0, tol=1.0e-10)
    dt, _ = o.cfl()
    h0, m0 = o.state()
    o.close()
    out = {}
    for prec in (PIP_FP64, PIP_MIXED):
        with capi.Context(s.overrides(precision=prec)) as c:
            c.upload(h0, m0)
            st, it, rr = c.conduction(dt)
            out[prec] = (st, it, rr, c.download())
    st64, it64, rr64, (h64, m64) = out[PIP_FP64]
    stmx, itmx, rrmx, (hmx, mmx) = out[PIP_MIXED]
    assert st64 == 0 and stmx == 0 and rr64 <= 1e-10 and rrmx <= 1e-10
    # the mixed context stores its state as an FP32 pair (~48 bits): compare the ion energy
    err = rel_l1(interior(mmx, s), interior(m64, s))[4]
    print("mixed vs fp64 ion energy", err, "iterations", it64, itmx)
    assert err <= 1e-8


def test_iteration_limit_is_reported(gpu_lib):
    s, o, Uh0, Um0 = kh_case(kapper=10.0, tol=1.0e-14)
    dt, _ = o.cfl()
    h0, m0 = o.state()
    o.close()
    with capi.Context(s.overrides(hc_max=3)) as c:
        c.upload(h0, m0)
        st, it, rr = c.conduction(dt)
        assert st == capi.PIP_ERR_ITER and it == 4 and rr > 1e-14
        st2, _, _ = c.run(nsteps=2)            # the run goes on, as the reference's does
        assert st2 == 0


def test_conduction_rejects_unsupported(gpu_lib):
    s, _, _ = ics.brio_wu(64, flag_heat=1, kapper=1.0)
    with pytest.raises(capi.PipError):
        capi.Context(s)
    s2, _, _ = ics.orszag_tang(32)
    with capi.Context(s2) as c:
        with pytest.raises(capi.PipError):
            c.conduction(1e-3)


def test_run_with_conduction_and_alpha_c_per_cell(gpu_lib):
    """Conduction after the stages with alpha_c per cell (set_collisional col_type 4)."""
    s, _, _ = ics.kelvin_helmholtz(48, 24, flag_heat=1, kapper=1.0, hc_error=1.0e-12,
                                   hc_max=2000, flag_col=5)
    Uh, Um = generic_state(s, 3)
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    st_o, t_o, n_o, _ = o.run(nsteps=12)
    oh, om = o.state()
    ac_o = o.alpha_c()
    o.close()
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, t, n = c.run(nsteps=12)
        gh, gm = c.download()
        ac_g = c.alpha_c()
    assert st_o == 0 and st == 0 and n == n_o == 12
    assert abs(t - t_o) <= 1e-12 * t_o
    assert max(rel_l1(interior(gh, s), interior(oh, s)).max(),
               rel_l1(interior(gm, s), interior(om, s)).max()) <= 1e-10
    assert np.abs(ac_g - ac_o).sum() <= 1e-10 * np.abs(ac_o).sum()


@pytest.mark.parametrize("precision", [PIP_FP64, PIP_MIXED])
def test_expired_staging_wait_is_reported_and_the_context_recovers(gpu_lib, precision):
    """A BiCGstab block whose mbarrier wait runs out (here: a limit of zero polls, so the
    first wait of every block runs out before its rows land) flags the solve instead of
    waiting on; the call reports it and the same context then solves normally."""
    import ctypes
    s, o, Uh0, Um0 = kh_case(kapper=1.0)
    dt, _ = o.cfl()
    h0, m0 = o.state()
    o.close()
    s = s.overrides(precision=precision)
    with capi.Context(s) as c:
        c.upload(h0, m0)
        ref = c.conduction(dt)
        c.pipbnd()
        rh, rm = c.download()
    L = capi.lib()
    with capi.Context(s) as c:
        c.set_hc_wait_limit(0)
        c.upload(h0, m0)
        it = ctypes.c_int()
        rr = ctypes.c_double()
        st = L.pip_conduction(c.h, float(dt), ctypes.byref(it), ctypes.byref(rr))
        assert st == capi.PIP_ERR_CUDA, capi.strerror(st)
        assert L.pip_last_cuda_error() == 702      # cudaErrorLaunchTimeout
        c.set_hc_wait_limit(-1)
        c.upload(h0, m0)
        again = c.conduction(dt)
        c.pipbnd()
        gh, gm = c.download()
    assert again == ref and ref[0] == 0
    assert np.array_equal(gh, rh) and np.array_equal(gm, rm)


@pytest.mark.parametrize("precision", [PIP_FP64, PIP_MIXED])
def test_device_loop_and_host_checked_groups_agree(gpu_lib, precision):
    """The BiCGstab iterations as one device-side loop (a conditional while node that the
    last kernel of an iteration ends) and in host-checked groups of four run the same
    kernels on the same buffers: identical iterates, counts and residuals, over several
    solves in a row, and the groups report an expired staging wait the same way."""
    import ctypes
    s, o, Uh0, Um0 = kh_case(kapper=1.0)
    dt, _ = o.cfl()
    h0, m0 = o.state()
    o.close()
    s = s.overrides(precision=precision)
    out = {}
    for loop in (True, False):
        with capi.Context(s) as c:
            c.set_hc_loop(loop)
            c.upload(h0, m0)
            res = [c.conduction(dt) for _ in range(3)]
            c.pipbnd()
            out[loop] = (res, c.download())
    (ra, (ah, am)), (rb, (bh, bm)) = out[True], out[False]
    assert ra == rb and all(r[0] == 0 and r[1] > 0 for r in ra)
    assert np.array_equal(ah, bh) and np.array_equal(am, bm)
    L = capi.lib()
    with capi.Context(s) as c:
        c.set_hc_loop(False)
        c.set_hc_wait_limit(0)
        c.upload(h0, m0)
        st = L.pip_conduction(c.h, float(dt), ctypes.byref(ctypes.c_int()),
                              ctypes.byref(ctypes.c_double()))
        assert st == capi.PIP_ERR_CUDA and L.pip_last_cuda_error() == 702
        assert L.pip_set_hc_loop(c.h, 2) == capi.PIP_ERR_PARAM
    plain, _, _ = ics.orszag_tang(16)
    with capi.Context(plain) as c:
        assert L.pip_set_hc_loop(c.h, 1) == capi.PIP_ERR_PARAM
