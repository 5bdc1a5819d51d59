"""set_IR type 4, the 6-level hydrogen model, on the CPU.

* The exponential-integral table: the oracle's regeneration of expintcalc/colexp.dat
  (colexpintcalc.f90) against the exponential integrals E_0, E_1, E_2 themselves (scipy) within
  the generator's own truncation, against a vectorised numpy trapezoid, and against the table the
  product library generates (bit for bit: same algorithm, same libm).
* The rates: the oracle's colrat, Gm_ion/Gm_rec and ion_pot after set_coefficients against an
  independent numpy transcription of get_col_ion_coeff / IRgetionpot (bit for bit).
* The excitation update of one stage against the numpy transcription (bit for bit).
* Invariants of whole runs: levels 1-5 sum to rho_n, Nexcite(6) = rho_i, the 1e-16 floor; the
  ionisation/recombination and excitation bounds lower dt when t_IR is large.
"""
import numpy as np
import pytest

import numpy_nlevel as NL
from oracle import oracle as O
from pip_b200 import capi, ics
from pip_b200.params import Settings

_TABLE = {}


def table(nsamps=100000):
    if nsamps not in _TABLE:
        O.set_threads(8)
        _TABLE[nsamps] = O.expint_table(nsamps)
    return _TABLE[nsamps]


def oracle_case(s, Uh, Um, nex, tab):
    o = O.Oracle(s, Uh, Um)
    o.set_nlevel(tab, deriv=s.nlev_deriv, n0fac=s.n0fac, f_p_ini=s.f_p_ini,
                 f_p_p_ini=s.f_p_p_ini)
    o.set_nexcite(nex)
    return o


def test_table_is_the_exponential_integrals():
    from scipy.special import expn
    t = table()
    assert t.shape == (100001, 4)
    y = t[:, 0]
    assert y[0] == pytest.approx(0.0627, rel=1e-3) and y[-1] == 108.0
    assert np.all(np.diff(y) > 0)
    for n in range(3):
        exact = np.exp(-y) / y if n == 0 else expn(n, y)
        rel = np.abs(t[:, n + 1] - exact) / exact
        # the trapezoid's step (1e-3) and its stop at 1e-4 of the first step bound the error
        assert rel.max() < 1.2e-3, (n, rel.max())
        assert np.median(rel) < 6e-4


def test_table_rows_match_a_vectorised_trapezoid():
    t = table()
    rows = np.r_[0, 1, 7, 1000, 5000, 20000, 60000, 99999, 100000]
    for n in range(3):
        ref = NL.trapezoid(t[rows, 0], float(n))
        np.testing.assert_allclose(t[rows, n + 1], ref, rtol=1e-13, atol=0)


def test_product_table_equals_the_oracle_table():
    a = capi.colexp_table(3000)
    b = O.expint_table(3000)
    assert a.shape == b.shape == (3001, 4)
    assert np.array_equal(a, b)


def set_ir_te(s, m):
    """Te_p that set_IR type 4 reads: get_Te_MHD after set_collisional's rewrite (flag_col
    >= 2), each rewrite taking the pressure from the energy as it stands."""
    gm = s.gm

    def kin(m):
        return 0.5 * ((m[1] * m[1] + m[2] * m[2] + m[3] * m[3]) / m[0] + m[5] * m[5] +
                      m[6] * m[6] + m[7] * m[7])

    e = m[4]
    for _ in range(2 if s.flag_col >= 2 else 1):
        pr = np.maximum((gm - 1.0) * (e - kin(m)), s.pr_lim)
        e = pr / (gm - 1.0) + kin(m)
    return 0.5 * gm * (pr / m[0])


def _tube(**kw):
    return ics.nlevel_tube(96, **kw)


@pytest.mark.parametrize("itype,flag_col", [(1, 1), (0, 1), (2, 3), (0, 2)])
def test_rates_against_numpy(itype, flag_col):
    tab = table()
    s, Uh, Um, nex = _tube(flag_ir_type=itype, flag_col=flag_col, beta=0.1)
    o = oracle_case(s, Uh, Um, nex, tab)
    o.coefficients()
    cr = o.colrat()[:, :, 0]
    gi, gr = [a[0] for a in o.ir_rates()]
    Uh2, Um2 = o.state()
    te_p = set_ir_te(s, Um[:, 0])
    if s.flag_col % 2 == 1:
        tfac = s.t_norm / (float(np.float32(5.0) / np.float32(3.0)) * s.f_p_p_ini / s.f_p_ini)
    else:
        tfac = s.beta / 2.0 * s.f_p_p_ini * 5.0 / 6.0 / s.f_p_ini
    m = Um2[:, 0]
    gm = s.gm
    R = NL.Rates(tab)
    ref = R.colrat(te_p * s.t_norm / tfac, m[0] * s.n_norm / s.n0fac)
    assert np.array_equal(cr, ref)
    # Gm_rec_ref: the rates at (T_norm, n_norm) with cell (1,1,1)'s populations
    cref = R.colrat(np.array([s.t_norm]), np.array([s.n_norm]))
    _, g0 = R.sums(cref, nex[:, 0, :1])
    assert o.gm_rec_ref == g0[0]
    si, sr = R.sums(ref, nex[:, 0])
    np.testing.assert_array_equal(gi, si / Uh2[0, 0] / o.gm_rec_ref * s.t_ir)
    np.testing.assert_array_equal(gr, sr / m[0] / o.gm_rec_ref * s.t_ir)
    if itype == 0:
        # the prologue's ion_pot comes from the reference-state rates (PIP_rot.f90:277)
        ip = NL.ion_pot(cref[..., :1] * np.ones_like(te_p), nex[:, 0], gm, s.t_norm, s.beta,
                        s.flag_col, o.gm_rec_ref, s.t_ir)
        np.testing.assert_array_equal(o.ion_pot()[0], ip)
    o.close()


@pytest.mark.parametrize("deriv", [0, 1, 4])
def test_one_stage_excitation_update_against_numpy(deriv):
    tab = table()
    s, Uh, Um, nex = _tube(nlev_deriv=deriv, t_ir=10.0)
    o = oracle_case(s, Uh, Um, nex, tab)
    o.prologue()
    nex0 = o.nexcite()
    dt = 2.0e-4
    o.stage(1, dt)      # set_IR of the stage, the stage, the update over dt/2
    cr = o.colrat()[:, :, 0]
    Uh1, Um1 = o.state()
    ref = NL.excitation_update_1d(nex0[:, 0], cr, Uh1[0, 0], Um1[0, 0], Uh1[1, 0],
                                  s.coordinates()[3], dt / 2.0, o.gm_rec_ref, s.t_ir, deriv)
    got = o.nexcite()[:, 0]
    m = s.margin[0]
    np.testing.assert_array_equal(got[:, m:-m], ref[:, m:-m])
    # bnd_energy: outflow (type 10) ghosts copy the first interior cell
    for g in range(m):
        np.testing.assert_array_equal(got[:, g], got[:, m])
        np.testing.assert_array_equal(got[:, -1 - g], got[:, -1 - m])
    o.close()


@pytest.mark.parametrize("itype", [0, 1])
def test_run_invariants(itype):
    tab = table()
    s, Uh, Um, nex = _tube(flag_ir_type=itype, t_ir=0.1)
    o = oracle_case(s, Uh, Um, nex, tab)
    o.prologue()
    st, t, n, _ = o.run(nsteps=40, max_hist=40)
    assert st == 0 and n == 40 and o.nlevel_status == 0
    Uh2, Um2 = o.state()
    nx = o.nexcite()
    m = s.margin[0]
    inner = (slice(None), 0, slice(m, -m))
    np.testing.assert_allclose(nx[:5].sum(0)[0, m:-m], Uh2[0, 0, m:-m], rtol=1e-14, atol=0)
    assert np.array_equal(nx[5][0, m:-m], Um2[0, 0, m:-m])
    assert nx[inner][:5].min() >= float(np.float32(1e-16))
    # the ions changed through ionisation/recombination as well as the flow
    assert np.isfinite(Uh2).all() and np.isfinite(Um2).all()
    o.close()


def test_ir_bounds_lower_dt():
    tab = table()
    dts = []
    for tir in (0.1, 100.0):
        s, Uh, Um, nex = _tube(flag_ir_type=0, t_ir=tir)
        o = oracle_case(s, Uh, Um, nex, tab)
        o.prologue()
        st, t, n, hist = o.run(nsteps=30, max_hist=30)
        assert st == 0
        dts.append(hist.min())
        o.close()
    assert dts[1] < 0.5 * dts[0]


def test_negative_rate_is_flagged():
    # a table whose integrals are negated makes the ionisation coefficients negative: the
    # reference stops there (PIP_rot.f90:546-557)
    tab = table(2000).copy()
    tab[:, 1:] = -tab[:, 1:]
    s, Uh, Um, nex = _tube()
    o = oracle_case(s, Uh, Um, nex, tab)
    o.coefficients()
    assert o.nlevel_status == 1
    o.close()


def test_settings():
    s, Uh, Um, nex = _tube()
    s.validate()
    for bad in (dict(n_levels=4), dict(flag_rad=2), dict(nlev_deriv=2),
                dict(flag_ir_type=3), dict(t_norm=0.0)):
        with pytest.raises(ValueError):
            s.overrides(**bad).validate()
    with pytest.raises(ValueError):
        Settings(flag_ir=2, flag_ir_type=0, t_norm=1e4, n_norm=1e16).validate()
    t = Settings.from_setting_text("5 :nlevels;\n1 :flag_rad;\n4 :flag_IR;\n0 :flag_IR_type;\n")
    assert (t.n_levels, t.flag_rad, t.flag_ir, t.flag_ir_type) == (5, 1, 4, 0)


def test_output_layout(tmp_path):
    from pip_b200 import output
    s, Uh, Um, nex = _tube(flag_ir_type=0)
    names = output.variables(s)
    i = names.index("rec")
    assert names[i + 1: i + 8] == ("nexcite1", "colrat11", "colrat12", "colrat13", "colrat14",
                                   "colrat15", "colrat16")
    assert names[i + 1 + 6 * 7] == "ion_loss" and names[-5:] == output.VAR_H
    rng = np.random.default_rng(3)
    shp = Uh.shape[1:]
    nl = dict(ion=rng.random(shp), rec=rng.random(shp), nexcite=nex,
              colrat=rng.random((6, 6) + shp), ion_loss=rng.random(shp))
    output.write_output(str(tmp_path), 2, s, 0.5, Uh, Um, nlevel=nl)
    d = output.read_output(output.file_stem(str(tmp_path), 2))
    assert np.array_equal(d["colrat34"][0], nl["colrat"][2, 3])
    assert np.array_equal(d["ion_loss"][0], nl["ion_loss"])
    assert np.array_equal(output.restart_nexcite(str(tmp_path), 2, s), nex)
    with pytest.raises(ValueError):
        output.write_output(str(tmp_path), 3, s, 0.5, Uh, Um)
