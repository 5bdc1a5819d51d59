"""Resistivity (flag_resi: resistive_flux, Solver_rot.f90:505-638, and cfl_resi,
Scheme_rot.f90:291-302) in the oracle, on the CPU.

The face terms are checked against a vectorised restatement of resistive_flux's flag_sch=0
branch with get_rotation (Util_rot.f90:148-236); the oracle's physics is pinned by the
resistive decay of a small sinusoidal field, whose rate the discrete operator fixes to
eta*sin(k dx)^2/dx^2 (eta*k^2 to second order).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from oracle_block import OracleBlock
from pip_b200 import decomp, ics, output
from pip_b200.params import PIP_MIXED, Settings
from resistive_cases import decay_case, decay_factor


def literal_resistive_terms(s, U_m, eta, direction):
    """F_m increments of resistive_flux for one direction, every face of the array."""
    ix, jx, _ = s.shape
    _, _, _, dx, dy, _ = s.coordinates()
    bx, by, bz = U_m[5], U_m[6], U_m[7]
    R = np.zeros((3, jx, ix))
    if s.ndim == 1:
        R[1, :, 1:-1] = -(bz[:, 2:] - bz[:, :-2]) / (2.0 * dx[1:-1])
        R[2, :, 1:-1] = (by[:, 2:] - by[:, :-2]) / (2.0 * dx[1:-1])
    else:
        dxc = dx[None, 1:-1]
        dyc = dy[1:-1, None]
        R[0, 1:-1, 1:-1] = (bz[2:, 1:-1] - bz[:-2, 1:-1]) / (2.0 * dyc)
        R[1, 1:-1, 1:-1] = -(bz[1:-1, 2:] - bz[1:-1, :-2]) / (2.0 * dxc)
        R[2, 1:-1, 1:-1] = ((by[1:-1, 2:] - by[1:-1, :-2]) / (2.0 * dxc)
                            - (bx[2:, 1:-1] - bx[:-2, 1:-1]) / (2.0 * dyc))
    ex, ey, ez = R[0] * eta, R[1] * eta, R[2] * eta
    d = {}
    if direction == 1:
        sl0, sl1 = (slice(None), slice(0, ix - 1)), (slice(None), slice(1, ix))
        d[4] = 0.25 * ((ey[sl1] + ey[sl0]) * (bz[sl0] + bz[sl1]) - (ez[sl0] + ez[sl1]) * (by[sl0] + by[sl1]))
        d[6] = -0.5 * (ez[sl0] + ez[sl1])
        d[7] = 0.5 * (ey[sl0] + ey[sl1])
    else:
        sl0, sl1 = (slice(0, jx - 1), slice(None)), (slice(1, jx), slice(None))
        d[4] = 0.25 * ((ez[sl1] + ez[sl0]) * (bx[sl0] + bx[sl1]) - (ex[sl0] + ex[sl1]) * (bz[sl0] + bz[sl1]))
        d[5] = 0.5 * (ez[sl0] + ez[sl1])
        d[7] = -0.5 * (ex[sl0] + ex[sl1])
    return d, sl0


@pytest.mark.parametrize("direction", [1, 2])
def test_face_terms_match_the_literal_restatement(direction):
    s, Uh, Um = ics.orszag_tang(24, flag_resi=1, eta_0=3e-3)
    eta = 3e-3 * (1.0 + np.random.default_rng(4).random(Uh.shape[1:]))
    o = O.Oracle(s, Uh, Um)
    o.set_resistivity(eta)
    Fh, Fm = o.flux(direction)
    o.close()
    o0 = O.Oracle(s, Uh, Um)                         # eta = 0: the ideal fluxes
    o0.set_resistivity(np.zeros_like(eta))
    Fh0, Fm0 = o0.flux(direction)
    o0.close()
    np.testing.assert_array_equal(Fh, Fh0)          # the neutrals have no resistive flux
    d, sl = literal_resistive_terms(s, Um, eta, direction)
    want = Fm0.copy()
    for n, inc in d.items():
        want[n][sl] = Fm0[n][sl] + inc
    np.testing.assert_array_equal(Fm, want)


def test_resistive_decay_rate():
    s, Uh, Um = decay_case(128, 1e-2)
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    st, t, n, _ = o.run(0, 1.0)
    _, om = o.state()
    o.close()
    assert st == 0 and t >= 1.0
    amp, want = decay_factor(s, om, t)
    assert abs(amp / want - 1.0) < 1e-5, (amp, want)
    # and eta*k^2 of the continuum to the discretisation's second order
    assert abs(amp / math.exp(-1e-2 * (2 * math.pi) ** 2 * t) - 1.0) < 1e-3


def test_cfl_resi_bound():
    """A large eta: dt is cfl_resi's safety*min(gmin)^2/eta."""
    s, Uh, Um = ics.orszag_tang(16, flag_resi=1, eta_0=10.0)
    o = O.Oracle(s, Uh, Um)
    dt, _ = o.cfl()
    o.close()
    _, _, _, dx, dy, dz = s.coordinates()
    m = s.margin
    g = min(dx[m[0]:-m[0]].min(), dy[m[1]:-m[1]].min(), dz[0])
    assert dt == s.safety * (g * g) / 10.0


def test_localised_field():
    s = Settings(ndim=2, ix0=16, jx0=16, start=(-1.0, -1.0, 0.0), flag_resi=11, eta_0=2.0,
                 debug_parameter=0.25)
    e = s.eta_field()
    x, y, _, _, _, _ = s.coordinates()
    for i, j in ((5, 9), (0, 0), (19, 3)):
        want = 2.0 * math.exp(-((x[i] / 0.8) ** 2 + ((y[j] - 0.25) / 0.8) ** 2))
        assert abs(e[j, i] / want - 1.0) < 1e-15
    assert Settings(flag_resi=1, eta_0=0.5).eta_field().min() == 0.5


@pytest.mark.parametrize("world", [2, 4])
def test_blocks_with_a_localised_field(world):
    """Decomposed oracle blocks with their parts of a localised eta field give the single
    domain's run bitwise."""
    s, Uh, Um = ics.kelvin_helmholtz(16, 16, flag_resi=11, eta_0=2e-3)
    eta = s.eta_field()
    o = O.Oracle(s, Uh, Um)
    o.set_resistivity(eta)
    st, t, n, hist = o.run(nsteps=5, max_hist=5)
    oh, om = o.state()
    o.close()
    engines = [OracleBlock(decomp.block_of(s, world, r), decomp.scatter(s, Uh, world, r),
                           decomp.scatter(s, Um, world, r),
                           eta=decomp.scatter(s, eta[None], world, r)[0]) for r in range(world)]
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    assert run.run(5) == 0
    states = [e.download() for e in engines]
    run.close()
    assert np.array_equal(np.array(run.dt_history), hist)
    assert np.array_equal(decomp.gather(s, [a for a, _ in states]), oh)
    assert np.array_equal(decomp.gather(s, [b for _, b in states]), om)


def test_settings_and_output(tmp_path):
    with pytest.raises(ValueError, match="flag_resi"):
        Settings(flag_resi=3).validate()
    with pytest.raises(ValueError, match="vd_cri"):
        Settings(flag_resi=32).validate()
    for v, want in ((2, 1), (12, 1), (21, 1), (22, 2), (32, 2)):
        p, _ = Settings(flag_resi=v, vd_cri=1.0).to_params()
        assert (p.flag_resi, p.resi_type) == (want, v // 10)
    with pytest.raises(ValueError, match="PIP_FP64"):
        Settings(flag_resi=1, precision=PIP_MIXED).validate()
    with pytest.raises(ValueError, match="conduction"):
        Settings(ndim=2, flag_resi=1, flag_heat=1).validate()
    s = Settings.from_setting_text("11:flag_resi;\n2.5d-3:eta_0;\n0.1:debug_parameter;\n")
    assert (s.flag_resi, s.eta_0, s.debug_parameter) == (11, 2.5e-3, 0.1)
    p, _ = s.to_params()
    assert p.flag_resi == 1 and p.eta_0 == 2.5e-3
    # def_varfiles' "et" and restart's read of it
    s, Uh, Um = ics.kelvin_helmholtz(16, 16, flag_resi=11, eta_0=1e-3)
    path = output.write_output(str(tmp_path), 1, s, 0.5, Uh, Um)
    names = [ln.split()[0] for ln in open(path[:-4] + ".idx")]
    assert names[7:9] == ["et", "ro_p"]
    np.testing.assert_array_equal(output.restart_resistivity(str(tmp_path), 1, s), s.eta_field())


# ------------------------------------------------------------ anomalous eta (flag_resi 2)

ANOMALOUS = [dict(flag_resi=22, eta_0=5e-3, j_cri=3.0),
             dict(flag_resi=32, eta_0=2e-2, vd_cri=150.0)]


@pytest.mark.parametrize("kw", ANOMALOUS)
def test_anomalous_eta_at_the_prologue_matches_the_restatement(kw):
    """set_resistivity resi_type 2 and 3 (Res_rot.f90:37-60) in the oracle against the
    vectorised restatement of Settings.eta_field, on the Orszag-Tang field, where both
    branches of each law occur."""
    s, Uh, Um = ics.orszag_tang(48, **kw)
    o = O.Oracle(s, Uh, Um)
    eta = o.resistivity()
    o.close()
    want = s.eta_field(Um)
    np.testing.assert_array_equal(eta, want)
    big = eta > kw["eta_0"] if kw["flag_resi"] == 22 else eta > 0.0
    assert 0.05 < big.mean() < 0.95


def _run(s, Uh, Um, nsteps):
    o = O.Oracle(s, Uh, Um)
    try:
        o.prologue()
        st, t, n, _ = o.run(nsteps, 0.0)
        h, m = o.state()
        return t, h, m
    finally:
        o.close()


def test_anomalous_eta_reduces_to_the_fixed_field_paths():
    """Per-stage eta whose switch never fires equals the fixed-field runs bit for bit: resi
    type 2 with j_cri beyond any current is uniform eta_0 (flag_resi 1), type 3 with vd_cri
    beyond any drift is eta = 0, the ideal run (flag_resi 0, two ghost layers)."""
    s2, Uh, Um = ics.orszag_tang(32, flag_resi=22, eta_0=2e-3, j_cri=1e30)
    s1 = s2.overrides(flag_resi=1)
    t2, h2, m2 = _run(s2, Uh, Um, 12)
    t1, h1, m1 = _run(s1, Uh, Um, 12)
    assert t2 == t1
    np.testing.assert_array_equal(h2, h1)
    np.testing.assert_array_equal(m2, m1)
    s3, Uh3, Um3 = ics.orszag_tang(32, flag_resi=32, eta_0=2e-3, vd_cri=1e30)
    s0, Uh0, Um0 = ics.orszag_tang(32)
    t3, h3, m3 = _run(s3, Uh3, Um3, 12)
    t0, h0, m0 = _run(s0, Uh0, Um0, 12)
    assert t3 == t0
    np.testing.assert_array_equal(h3[:, 3:-3, 3:-3], h0[:, 2:-2, 2:-2])
    np.testing.assert_array_equal(m3[:, 3:-3, 3:-3], m0[:, 2:-2, 2:-2])


def test_anomalous_eta_lowers_the_time_increment():
    """Where cfl_resi's bound of the last stage's eta is below the step's dt, the time loop
    advances time by the bound (main.f90:47,58, through cfl_resi's write of the global dt):
    time after the step = time before + min(dt, bound of the new eta)."""
    # type 2 switches eta to 11 eta_0 when a cell's current first passes j_cri: from then
    # on the bound of the new eta lies below the step's dt
    s, Uh, Um = ics.orszag_tang(32, flag_resi=22, eta_0=0.03, j_cri=5.5)
    o = O.Oracle(s, Uh, Um)
    try:
        o.prologue()
        lowered = 0
        for _ in range(30):
            t0 = o.time
            dt, _ = o.cfl()       # the step's dt (the run's own cfl gives the same)
            st, t1, n, _ = o.run(1, 0.0)
            assert st == 0 and n == 1
            bound = _bound(s, o.resistivity())
            assert t1 - t0 == pytest.approx(min(dt, bound), rel=1e-12)
            lowered += bound < dt
        assert lowered > 0
    finally:
        o.close()


def _bound(s, eta):
    m = s.margin
    _, _, _, dx, dy, dz = s.coordinates()
    gmin = np.minimum(np.minimum(dx[None, :], dy[:, None]), dz[0])
    b = s.safety * (gmin * gmin) / np.maximum(eta, 1e-8)
    return float(b[m[1]:-m[1], m[0]:-m[0]].min())
