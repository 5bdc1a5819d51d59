"""set_IR types 1-3 (PIP_rot.f90:134-228: the Jeffery formulation and the Popescu et al.
2019 rates) in the oracle, on the CPU: the rates after set_coefficients against a vectorised
restatement written from the Fortran (its single-precision literals rounded to float), the
energy rewrite of get_Te, the cfl bound and a decomposed run."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle_block import OracleBlock
from pip_b200 import decomp, ics, output
from pip_b200.params import (PIP_IR_JEFFERY, PIP_IR_POPESCU, PIP_IR_POPESCU_EQ, PIP_MIXED,
                             Settings)


def case(law, **kw):
    return ics.kelvin_helmholtz(32, 16, flag_ir=law, t_norm=1.5e4, n_norm=1.0e11, t_ir=10.0, **kw)


def literal_rates(s, U_m):
    """Gm_ion, Gm_rec of set_IR type 1, 2 or 3 after get_Te_MHD, whole-array, Fortran order."""
    gm = s.gm
    m2 = U_m[1] * U_m[1] + U_m[2] * U_m[2] + U_m[3] * U_m[3]
    pr = (gm - 1.0) * (U_m[4] - 0.5 * ((m2 / U_m[0] + U_m[5] * U_m[5]) + U_m[6] * U_m[6]
                                       + U_m[7] * U_m[7]))
    if pr.min() <= s.pr_lim:
        pr = np.maximum(pr, s.pr_lim)
    Te_p = 0.5 * gm * (pr / U_m[0])
    T0, n0, t_ir = s.t_norm, s.n_norm, s.t_ir
    r = lambda x: float(np.float32(x))                  # a REAL*4 literal
    if s.flag_ir == PIP_IR_JEFFERY:
        factor = np.exp(-13.2 / (T0 / 11605.0))
        factor2 = r(2.7) * (13.2 * 11605.0) ** -2.0 * T0 ** (1.0 / 2.0) * n0
        factor3 = r(5.6e-16) * (13.2 * 11605.0) ** -2.0 * T0 ** -1.0 * n0 ** 2.0
        rec_fac = factor2 / factor3
        ion_fac = factor3 / t_ir
        Gm_rec = Te_p ** -0.5 * U_m[0] ** 2.0 * rec_fac * ion_fac
        Gm_ion = Te_p ** 0.5 * U_m[0] * factor ** (1.0 / Te_p) * ion_fac
        return Gm_ion, Gm_rec
    Te_0 = T0 / r(1.1604e4)
    if s.flag_ir == PIP_IR_POPESCU:
        rec_fac = r(2.6e-19) * (n0 * r(1.0e6)) / np.sqrt(Te_0) * t_ir
        Gm_rec = U_m[0] / np.sqrt(Te_p) * rec_fac
        Gm_ion = ((n0 * r(1.0e6) * U_m[0]) * r(2.91e-14) * np.exp(-13.6 / Te_0 / Te_p)
                  * (13.6 / Te_0 / Te_p) ** 0.39 / (0.232 + 13.6 / Te_0 / Te_p) * t_ir)
        return Gm_ion, Gm_rec
    rec_fac = r(2.6e-19) * (n0 * r(1.0e6)) / np.sqrt(Te_0)
    ioneq = (r(2.6e-19) / np.sqrt(Te_0)) / (r(2.91e-14) / (0.232 + 13.6 / Te_0)
                                             * (13.6 / Te_0) ** 0.39 * np.exp(-13.6 / Te_0))
    f_n = ioneq / (ioneq + 1.0)
    f_p = 1.0 - f_n
    f_p_p = 2.0 * f_p / (f_n + 2.0 * f_p)
    if s.flag_col % 2 == 1:
        tfac = 0.5 * f_p_p / f_p
    else:
        tfac = s.beta / 2.0 * f_p_p * 5.0 / 6.0 / f_p
    Gm_rec = U_m[0] / np.sqrt(Te_p) * t_ir / f_p * np.sqrt(tfac)
    Gm_ion = (r(2.91e-14) * (n0 * r(1.0e6)) * U_m[0] * np.exp(-13.6 / Te_0 / Te_p * tfac)
              * (13.6 / Te_0 / Te_p * tfac) ** 0.39)
    Gm_ion = Gm_ion / (0.232 + 13.6 / Te_0 / Te_p * tfac) / rec_fac / f_p * t_ir
    return Gm_ion, Gm_rec


@pytest.mark.parametrize("law,flag_col", [(PIP_IR_JEFFERY, 1), (PIP_IR_POPESCU, 1),
                                          (PIP_IR_POPESCU_EQ, 1), (PIP_IR_POPESCU_EQ, 4)])
def test_rates_match_the_literal_restatement(law, flag_col):
    s, Uh, Um = case(law, flag_col=flag_col)
    o = O.Oracle(s, Uh, Um)
    try:
        o.coefficients()
        ion, rec = o.ir_rates()
        oh, om = o.state()
    finally:
        o.close()
    want_ion, want_rec = literal_rates(s, Um)
    assert np.all(rec > 0.0) and np.all(ion > 0.0)
    # exp and x**0.39 of numpy against libm: a few ulp
    np.testing.assert_allclose(rec, want_rec, rtol=1e-15, atol=0.0)
    np.testing.assert_allclose(ion, want_ion, rtol=1e-14, atol=0.0)
    # the output writer's rates are these (from the state the rates were taken from)
    w_ion, w_rec = output.ir_rates(s, om)
    np.testing.assert_allclose(w_rec, rec, rtol=1e-15, atol=0.0)
    np.testing.assert_allclose(w_ion, ion, rtol=1e-14, atol=0.0)
    # get_Te rewrote the energies only
    np.testing.assert_array_equal(om[[0, 1, 2, 3, 5, 6, 7]], Um[[0, 1, 2, 3, 5, 6, 7]])
    np.testing.assert_allclose(om[4], Um[4], rtol=1e-14)


@pytest.mark.parametrize("law", [PIP_IR_JEFFERY, PIP_IR_POPESCU_EQ])
def test_cfl_bound_and_run(law):
    s, Uh, Um = case(law)
    o = O.Oracle(s, Uh, Um)
    try:
        dt, _ = o.cfl()
        ion, rec = o.ir_rates()
        bound = min(s.safety, 0.1) / max(ion.max(), rec.max(), 1e-5)
        assert dt <= bound * (1 + 1e-15)
        st, t, n, _ = o.run(nsteps=20)
        assert st == 0 and n == 20 and not o.has_nan()
    finally:
        o.close()


@pytest.mark.parametrize("law", [PIP_IR_JEFFERY, PIP_IR_POPESCU, PIP_IR_POPESCU_EQ])
def test_blocks_match_single_domain(law):
    s, Uh, Um = case(law, flag_col=5)
    o = O.Oracle(s, Uh, Um)
    st, t, n, hist = o.run(nsteps=5, max_hist=5)
    oh, om = o.state()
    o.close()
    engines = [OracleBlock(decomp.block_of(s, 2, r), decomp.scatter(s, Uh, 2, r),
                           decomp.scatter(s, Um, 2, r)) for r in range(2)]
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    assert run.run(5) == 0
    states = [e.download() for e in engines]
    run.close()
    assert np.array_equal(np.array(run.dt_history), hist)
    assert np.array_equal(decomp.gather(s, [a for a, _ in states]), oh)
    assert np.array_equal(decomp.gather(s, [b for _, b in states]), om)


def test_settings():
    with pytest.raises(ValueError, match="T_norm"):
        Settings(flag_ir=3).validate()
    with pytest.raises(ValueError, match="PIP_FP64"):
        Settings(flag_ir=2, t_norm=1e4, n_norm=1e11, precision=PIP_MIXED).validate()
    s = Settings.from_setting_text("3:flag_IR;\n1.5d4:T_norm;\n1d11:n_norm;\n")
    assert (s.flag_ir, s.t_norm, s.n_norm) == (3, 1.5e4, 1e11)
    p, _ = s.to_params()
    assert p.t_norm == 1.5e4 and p.n_norm == 1e11


def test_type3_equilibrium_has_no_mass_exchange():
    """set_IR type 3 is scaled to the ionisation equilibrium of T_norm: at the ion
    temperature tfac (code units) and rho_n/rho_i = ioneq the ionisation and recombination
    mass rates cancel (source_PIP's IR block, PIP_rot.f90:1370-1376)."""
    s, _, _ = case(PIP_IR_POPESCU_EQ)
    f32 = lambda x: float(np.float32(x))
    Te_0 = s.t_norm / f32(1.1604e4)
    ioneq = (f32(2.6e-19) / np.sqrt(Te_0)) / (f32(2.91e-14) / (0.232 + 13.6 / Te_0)
                                               * (13.6 / Te_0) ** 0.39 * np.exp(-13.6 / Te_0))
    f_n = ioneq / (ioneq + 1.0)
    f_p = 1.0 - f_n
    tfac = 0.5 * (2.0 * f_p / (f_n + 2.0 * f_p)) / f_p          # flag_col 1
    ix, jx, _ = s.shape
    ro_i = 0.3
    ro_n = ioneq * ro_i
    p_i = tfac * ro_i / (0.5 * s.gm)                          # Te_p = 0.5*gm*p/ro = tfac
    zero = np.zeros((jx, ix))
    Uh = ics.pv2cq_hd(s, ro_n + zero, zero, zero, zero, 0.4 + zero)
    Um = ics.pv2cq_mhd(s, ro_i + zero, zero, zero, zero, p_i + zero, 0.1 + zero, zero, zero)
    o = O.Oracle(s.overrides(col=0.0), Uh, Um)
    try:
        o.coefficients()
        ion, rec = o.ir_rates()
        S_h, S_m = o.source(1e-3)
    finally:
        o.close()
    scale = rec * ro_i
    assert np.all(np.abs(S_m[0]) <= 1e-12 * scale)      # rec*ro_i - ion*ro_n = 0
    np.testing.assert_allclose(ion * ro_n, rec * ro_i, rtol=1e-12)
