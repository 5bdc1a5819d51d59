"""set_IR type 4, the 6-level hydrogen model, on the device through the C ABI, against the
oracle (PIP_rot.f90:232-311,361-616,919-946,1026-1235; Scheme_rot.f90:315-335,692-736,
1002-1049).

The rates go through exp, log and pow, whose last bits differ between CUDA and the host's
libm, so no run here is bitwise: states, populations, rates and time are held to 1e-10
relative L1 per variable (the drop-in tolerance), single calls to 1e-12.  The table is the
product's regeneration of expintcalc/colexp.dat, which equals the oracle's bit for bit
(tests/test_nlevel_host.py).
"""
import numpy as np
import pytest
import torch

from helpers import interior, rel_l1
from oracle import oracle as O
from pip_b200 import capi, ics

pytestmark = pytest.mark.gpu

TOL = 1e-10
TOL_CALL = 1e-12
_TAB = {}


def table(n=100000):
    if n not in _TAB:
        _TAB[n] = capi.colexp_table(n)
    return _TAB[n]


def setup_gpu(c, s, Uh, Um, nex, tab):
    c.upload(Uh, Um)
    c.set_nlevel(tab)          # the settings' n_levels, deriv, n0fac, f_p_ini, f_p_p_ini
    c.set_nexcite(nex)


def setup_orc(s, Uh, Um, nex, tab):
    O.set_threads(8)
    o = O.Oracle(s, Uh, Um)
    o.set_nlevel(tab, deriv=s.nlev_deriv, n0fac=s.n0fac, f_p_ini=s.f_p_ini,
                 f_p_p_ini=s.f_p_p_ini)
    o.set_nexcite(nex)
    return o


def run_pair(s, Uh, Um, nex, nsteps, tab=None):
    tab = table() if tab is None else tab
    with capi.Context(s) as c:
        setup_gpu(c, s, Uh, Um, nex, tab)
        c.prologue()
        g = c.run(nsteps, check=False)
        gh, gm = c.download()
        gx = c.nexcite()
        gcr = c.colrat()
        gip = c.ion_pot()
        gref = c.gm_rec_ref()
    o = setup_orc(s, Uh, Um, nex, tab)
    o.prologue()
    ost, ot, on, _ = o.run(nsteps=nsteps)
    oh, om = o.state()
    ox, ocr, oip, oref = o.nexcite(), o.colrat(), o.ion_pot(), o.gm_rec_ref
    o.close()
    return dict(g=g, o=(ost, ot, on), gh=gh, gm=gm, oh=oh, om=om, gx=gx, ox=ox, gcr=gcr,
                ocr=ocr, gip=gip, oip=oip, gref=gref, oref=oref)


def check(r, s, tol=TOL):
    gst, gt, gn = r["g"]
    ost, ot, on = r["o"]
    assert gst == 0 and ost == 0 and gn == on
    assert abs(gt - ot) <= tol * ot
    assert abs(r["gref"] - r["oref"]) <= 1e-14 * r["oref"]
    e = max(rel_l1(interior(r["gh"], s), interior(r["oh"], s)).max(),
            rel_l1(interior(r["gm"], s), interior(r["om"], s)).max())
    assert e <= tol, e
    ex = rel_l1(interior(r["gx"], s), interior(r["ox"], s)).max()
    assert ex <= tol, ex
    ecr = rel_l1(r["gcr"].reshape(36, *r["gcr"].shape[2:]), r["ocr"].reshape(36, *r["ocr"].shape[2:]))
    assert ecr.max() <= tol, ecr.max()
    return e, ex


@pytest.mark.parametrize("exact", [1, 0])
@pytest.mark.parametrize("itype,deriv", [(1, 1), (0, 4), (2, 0)])
def test_tube_against_oracle(exact, itype, deriv):
    s, Uh, Um, nex = ics.nlevel_tube(256, flag_ir_type=itype, nlev_deriv=deriv, t_ir=0.1,
                                     fp_exact=exact)
    r = run_pair(s, Uh, Um, nex, 40)
    check(r, s)
    if itype == 0:
        assert rel_l1(r["gip"][None], r["oip"][None]).max() <= TOL


def test_tube_ir_bounds_set_dt():
    # t_IR = 100: cfl_pip_ir's and cfl_pip_ir_nexcite's bounds take over from the CFL
    s, Uh, Um, nex = ics.nlevel_tube(256, flag_ir_type=0, nlev_deriv=1, t_ir=100.0, fp_exact=1)
    r = run_pair(s, Uh, Um, nex, 30)
    check(r, s)
    s1, Uh1, Um1, nex1 = ics.nlevel_tube(256, flag_ir_type=0, nlev_deriv=1, t_ir=0.1, fp_exact=1)
    r1 = run_pair(s1, Uh1, Um1, nex1, 30)
    assert r["g"][1] < 0.5 * r1["g"][1]


@pytest.mark.parametrize("exact,deriv,flag_col", [(1, 4, 1), (0, 1, 3)])
def test_orszag_tang_against_oracle(exact, deriv, flag_col):
    s, Uh, Um, nex = ics.nlevel_orszag_tang(64, nlev_deriv=deriv, flag_col=flag_col, beta=0.1,
                                            flag_ir_type=0, t_ir=1.0, fp_exact=exact)
    r = run_pair(s, Uh, Um, nex, 20)
    check(r, s)


def test_single_calls_against_oracle():
    s, Uh, Um, nex = ics.nlevel_tube(128, flag_ir_type=0, nlev_deriv=1, t_ir=1.0, fp_exact=1)
    tab = table()
    o = setup_orc(s, Uh, Um, nex, tab)
    with capi.Context(s) as c:
        setup_gpu(c, s, Uh, Um, nex, tab)
        dt, cm = c.cfl()
        odt, ocm = o.cfl()
        assert abs(dt - odt) <= TOL_CALL * odt
        o.cmax = ocm
        gS = c.source_pip(dt * 0.5)
        oS = o.source(odt * 0.5)
        for a, b in zip(gS, oS):
            assert rel_l1(a, b).max() <= TOL_CALL
        assert rel_l1(c.ion_pot()[None], o.ion_pot()[None]).max() <= TOL_CALL
        gcr, ocr = c.colrat(), o.colrat()
        assert rel_l1(gcr.reshape(36, -1), ocr.reshape(36, -1)).max() <= TOL_CALL
        # one host-given step
        c.run_solver(dt)
        o.run_solver(odt)
        gh, gm = c.download()
        oh, om = o.state()
        assert max(rel_l1(gh, oh).max(), rel_l1(gm, om).max()) <= TOL_CALL
        assert rel_l1(c.nexcite(), o.nexcite()).max() <= TOL_CALL
    o.close()


def test_api_rules():
    s, Uh, Um, nex = ics.nlevel_tube(64)
    tab = table()
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        with pytest.raises(capi.PipError) as e:
            c.cfl()                                 # no pip_set_nlevel yet
        assert e.value.code == capi.PIP_ERR_STATE
        for bad in (dict(n_levels=4), dict(flag_rad=2), dict(deriv=2)):
            with pytest.raises(capi.PipError) as e:
                c.set_nlevel(tab, **bad)
            assert e.value.code == capi.PIP_ERR_PARAM
        with pytest.raises(capi.PipError):
            c.set_nlevel(tab[::-1])                 # abscissae must increase
        c.set_nlevel(tab)
        c.set_nexcite(nex)
        with pytest.raises(capi.PipError) as e:
            c.set_neighbors([1, -1, -1, -1])         # single rank only
        assert e.value.code == capi.PIP_ERR_PARAM
        with pytest.raises(capi.PipError) as e:
            c.dev_begin(nsteps=1)
        assert e.value.code == capi.PIP_ERR_PARAM
        c.prologue()
        st, t, n = c.run(5)
        assert st == 0 and n == 5
    s2, Uh2, Um2 = ics.brio_wu(64)
    with capi.Context(s2) as c:
        with pytest.raises(capi.PipError) as e:
            c.set_nlevel(tab)                       # not a set_IR type 4 context
        assert e.value.code == capi.PIP_ERR_PARAM


def test_negative_rate_stops_the_run():
    # negated integrals make the ionisation coefficients negative, where the reference stops
    tab = table(2000).copy()
    tab[:, 1:] = -tab[:, 1:]
    s, Uh, Um, nex = ics.nlevel_tube(64)
    with capi.Context(s) as c:
        setup_gpu(c, s, Uh, Um, nex, tab)
        with pytest.raises(capi.PipError) as e:
            c.prologue()
        assert e.value.code == capi.PIP_ERR_RATE
        st, t, n = c.run(3, check=False)
        assert st == capi.PIP_ERR_RATE and n == 0     # stopped before the first step
    # the device stays usable
    s, Uh, Um, nex = ics.nlevel_tube(64)
    with capi.Context(s) as c:
        setup_gpu(c, s, Uh, Um, nex, table())
        c.prologue()
        assert c.run(3)[0] == 0
    torch.cuda.synchronize()


def test_output_datasets(tmp_path):
    from pip_b200 import output
    s, Uh, Um, nex = ics.nlevel_tube(128, flag_ir_type=0, fp_exact=1)
    with capi.Context(s) as c:
        setup_gpu(c, s, Uh, Um, nex, table())
        c.prologue()
        st, last, t = output.run_with_output(c, s, str(tmp_path), dtout=0.002, tend=0.004)
        assert st == 0 and last == 2
        ion, rec = c.ir_rates()
        nx, cr, ip = c.nexcite(), c.colrat(), c.ion_pot()
        gh, gm = c.download()
    d = output.read_output(output.file_stem(str(tmp_path), 2))
    assert d["time"] == t
    assert np.array_equal(d["ion"][0], ion) and np.array_equal(d["rec"][0], rec)
    assert np.array_equal(d["ion_loss"][0], ip)
    assert np.array_equal(d["nexcite3"][0], nx[2]) and np.array_equal(d["colrat52"][0], cr[4, 1])
    assert np.array_equal(output.restart_nexcite(str(tmp_path), 2, s), nx)
    assert np.array_equal(d["ro_n"][0], gh[0])
