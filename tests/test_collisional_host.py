"""Temperature- and drift-dependent collision coefficient (flag_col 2..7) on the CPU.

The oracle's set_collisional is checked against a vectorised restatement written from
PIP_rot.f90:44-97 (col_type 1..6) with get_Te_MHD / get_Te_HD (Scheme_rot.f90:83-128) and
get_vel_diff (:988-999); the Settings checks mirror the C ABI's parameter validation.
"""
import numpy as np
import pytest

from oracle import oracle as O
from pip_b200 import ics
from pip_b200.params import PIP_MIXED, Settings

PI = 3.1415926535897932  # Parameters.f90:2


def literal_set_collisional(s, U_h, U_m, col_type):
    """Whole-array form of set_collisional: returns (ac, rewritten U_h, rewritten U_m)."""
    gm = s.gm
    U_h = U_h.copy()
    U_m = U_m.copy()
    m2 = U_m[1] * U_m[1] + U_m[2] * U_m[2] + U_m[3] * U_m[3]
    pr = (gm - 1.0) * (U_m[4] - 0.5 * ((m2 / U_m[0] + U_m[5] * U_m[5]) + U_m[6] * U_m[6]
                                       + U_m[7] * U_m[7]))
    if pr.min() <= s.pr_lim:
        pr = np.maximum(pr, s.pr_lim)
    U_m[4] = pr / (gm - 1.0) + 0.5 * ((m2 / U_m[0] + U_m[5] * U_m[5]) + U_m[6] * U_m[6]
                                      + U_m[7] * U_m[7])
    te_m = 0.5 * gm * (pr / U_m[0])
    n2 = U_h[1] * U_h[1] + U_h[2] * U_h[2] + U_h[3] * U_h[3]
    pr = (gm - 1.0) * (U_h[4] - 0.5 * n2 / U_h[0])
    if pr.min() <= s.pr_lim:
        pr = np.maximum(pr, s.pr_lim)
    U_h[4] = pr / (gm - 1.0) + 0.5 * (n2 / U_h[0])
    te_h = gm * (pr / U_h[0])
    vd = [U_h[k] / U_h[0] - U_m[k] / U_m[0] for k in (1, 2, 3)]
    v2 = vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]
    T = te_h + te_m
    col, beta = s.col, s.beta
    a = col * np.sqrt(T / 2.0)
    if col_type == 1:
        return a / np.sqrt(beta / 2.0 * gm), U_h, U_m
    if col_type == 2:
        return a, U_h, U_m
    a = a * np.sqrt(1.0 + 9.0 * PI / 64.0 * gm / 2.0 * v2 / T)
    if col_type == 3:
        return a / np.sqrt(beta / 2.0 * gm), U_h, U_m
    if col_type == 4:
        return a, U_h, U_m
    if col_type == 5:
        return (a / np.sqrt(beta / 2.0 * gm)
                * ((beta / 2.0 * gm) / T / 2.0 + gm * PI / 16.0 * v2) ** 0.125), U_h, U_m
    return a / (T / 2.0 + gm * PI / 16.0 * v2) ** 0.125, U_h, U_m


def drifting_state(kind, flag_col, seed):
    if kind == "ot":
        s, U_h, U_m = ics.orszag_tang(24, flag_col=flag_col, fp_exact=1)
    else:
        s, U_h, U_m = ics.brio_wu(96, flag_col=flag_col, fp_exact=1)
    rng = np.random.default_rng(seed)
    # a neutral drift and temperature spread so every term of alpha_c matters
    U_h = U_h.copy()
    U_h[1:4] += 0.3 * U_h[0] * rng.standard_normal(U_h[1:4].shape)
    U_h[4] *= 1.0 + 0.2 * rng.random(U_h[4].shape)
    return s, U_h, U_m


@pytest.mark.parametrize("kind", ["ot", "bw"])
@pytest.mark.parametrize("flag_col", [2, 3, 4, 5, 6, 7])
def test_alpha_c_matches_the_literal_formulas(kind, flag_col):
    s, U_h, U_m = drifting_state(kind, flag_col, 11 * flag_col)
    o = O.Oracle(s, U_h, U_m)
    try:
        a = o.alpha_c()
        oh, om = o.state()
    finally:
        o.close()
    ra, rh, rm = literal_set_collisional(s, U_h, U_m, flag_col - 1)
    assert a.shape == ra.shape and np.all(np.isfinite(a)) and a.min() > 0.0
    if flag_col in (6, 7):
        # x**0.125: numpy's vectorised pow and libm's may differ in the last bit
        np.testing.assert_allclose(a, ra, rtol=4e-16, atol=0.0)
    else:
        np.testing.assert_array_equal(a, ra)
    # get_Pr_HD / get_Pr_MHD rewrite the energies (and nothing else)
    np.testing.assert_array_equal(oh, rh)
    np.testing.assert_array_equal(om, rm)


def test_constant_alpha_c_field():
    s, U_h, U_m = ics.orszag_tang(16, fp_exact=1)
    o = O.Oracle(s, U_h, U_m)
    try:
        a = o.alpha_c()
        oh, om = o.state()
    finally:
        o.close()
    assert np.all(a == s.col)
    np.testing.assert_array_equal(oh, U_h)   # flag_col 1 leaves the state alone
    np.testing.assert_array_equal(om, U_m)


def test_col_type_2_at_unit_temperature_is_col():
    """col_type 2: alpha_c = col*sqrt((Te_h+Te_m)/2) = col when Te_h + Te_m = 2."""
    s, U_h, U_m = ics.orszag_tang(16, flag_col=3, fp_exact=1)
    gm = s.gm
    U_h = U_h.copy()
    U_m = U_m.copy()
    # Te_h = gm*p_h/ro_h = 1 and Te_m = 0.5*gm*p_m/ro_m = 1 at rest, without field
    U_h[1:4] = 0.0
    U_m[1:4] = 0.0
    U_m[5:8] = 0.0
    U_h[0] = 1.0
    U_m[0] = 1.0
    U_h[4] = (1.0 / gm) / (gm - 1.0)
    U_m[4] = (2.0 / gm) / (gm - 1.0)
    o = O.Oracle(s, U_h, U_m)
    try:
        a = o.alpha_c()
    finally:
        o.close()
    np.testing.assert_allclose(a, s.col, rtol=1e-15)


def test_stages_recompute_alpha_c():
    """A step with flag_col >= 2 leaves the alpha_c of its second stage's input state."""
    s, U_h, U_m = drifting_state("ot", 5, 3)
    o = O.Oracle(s, U_h, U_m)
    try:
        dt, cm = o.cfl()
        o.cmax = cm
        o.stage(1, dt)
        Uh1, Um1 = o.state()
        o.stage(2, dt)
        a = o.alpha_c()
    finally:
        o.close()
    ra, _, _ = literal_set_collisional(s, Uh1, Um1, 4)
    np.testing.assert_array_equal(a, ra)


def test_variable_alpha_c_bounds_dt():
    """cfl_pn_col with the alpha_c field: dt <= min(safety,0.3)/max(rho*alpha_c)."""
    s, U_h, U_m = drifting_state("ot", 4, 5)
    o = O.Oracle(s, U_h, U_m)
    try:
        a = o.alpha_c()
        oh, om = o.state()
        dt, _ = o.cfl()
    finally:
        o.close()
    bound = min(s.safety, 0.3) / max((om[0] * a).max(), (oh[0] * a).max())
    assert dt <= bound * (1 + 1e-15)


def test_settings_validation():
    s = Settings(flag_col=8)
    with pytest.raises(ValueError, match="flag_col"):
        s.validate()
    with pytest.raises(ValueError, match="PIP_FP64"):
        Settings(flag_col=3, precision=PIP_MIXED).validate()
    with pytest.raises(ValueError, match="beta"):
        Settings(flag_col=2, beta=0.0).validate()
    Settings(flag_col=3, beta=0.0).validate()       # col_type 2 does not use beta
    for fc in range(1, 8):
        Settings(flag_col=fc).validate()


def test_setting_file_reads_beta():
    s = Settings.from_setting_text("0.25:beta; initial plasma beta\n4:flag_col;\n")
    assert s.beta == 0.25 and s.flag_col == 4
    p, _ = s.to_params()
    assert p.beta == 0.25
