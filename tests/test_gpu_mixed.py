"""FP32-mixed form against the plain FP64 path: relative L1 per variable <= 1e-5."""
import numpy as np
import pytest

from helpers import interior, rel_l1
from pip_b200 import capi, ics
from pip_b200.params import PIP_MIXED

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-5


def run(s, Uh, Um, nsteps=0, t_end=0.0):
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, t, n = c.run(nsteps, t_end)
        assert st == 0
        return (t, n) + c.download()


def compare(s, Uh, Um, nsteps=0, t_end=0.0):
    a = run(s, Uh, Um, nsteps, t_end)
    b = run(s.overrides(precision=PIP_MIXED), Uh, Um, nsteps, t_end)
    err_h = rel_l1(interior(b[2], s), interior(a[2], s))
    err_m = rel_l1(interior(b[3], s), interior(a[3], s))
    return a, b, err_h, err_m


# The Dedner potential psi does not meet the 1e-5 bar in this form, and no form that rounds
# B to FP32 at every step can: test_psi_amplifies_white_noise_in_b shows the plain FP64
# path itself moving psi by >1e-4 relative L1 from a one-time 1e-10 perturbation of B.
# psi is ~1e-4 of |B| in size, and the grid-scale noise FP32 rounding puts into div B at
# every step drives it.  Measured on OT 1024^2 after 2000 steps: psi 4e-3 while the 13
# physical fields (8 MHD, 5 hydro) stay at ~5e-7.  psi is held to the measured level.
TOL_PSI = 1e-2


def test_mixed_orszag_tang(gpu_lib):
    s, Uh, Um = ics.orszag_tang(128)
    a, b, eh, em = compare(s, Uh, Um, nsteps=300)
    assert a[1] == b[1] == 300
    assert abs(a[0] - b[0]) <= 1e-5 * a[0]
    # vz / bz / mz stay exactly zero in this 2D problem; the others carry the check
    physical = max(eh.max(), em[:8].max())
    assert physical <= TOL_MIXED, (eh, em)
    assert em[8] <= TOL_PSI, em



def test_psi_amplifies_white_noise_in_b(gpu_lib):
    """The plain FP64 path alone, OT 1024^2: a one-time white relative perturbation of 1e-10
    of Bx and By moves psi by more than 1e-4 relative L1 within 10 steps (the 13 physical
    fields move by less than 1e-9).  The rounding-only change of the FMA-free build keeps
    psi within 1e-7 over the same steps."""
    s, Uh, Um = ics.orszag_tang(1024)
    rng = np.random.default_rng(7)
    Up = Um.copy()
    for n in (5, 6):
        Up[n] *= 1.0 + 1e-10 * rng.uniform(-1.0, 1.0, size=Up[n].shape)
    a = run(s, Uh, Um, nsteps=10)
    b = run(s, Uh, Up, nsteps=10)
    c = run(s.overrides(fp_exact=1), Uh, Um, nsteps=10)
    em = rel_l1(interior(b[3], s), interior(a[3], s))
    eh = rel_l1(interior(b[2], s), interior(a[2], s))
    print("psi after a 1e-10 B perturbation: %.3e; others max %.3e"
          % (em[8], max(eh.max(), em[:8].max())))
    assert em[8] > 1e-4
    assert max(eh.max(), em[:8].max()) < 1e-9
    assert rel_l1(interior(c[3], s), interior(a[3], s))[8] < 1e-7


def test_mixed_brio_wu(gpu_lib):
    s, Uh, Um = ics.brio_wu(1024)
    a, b, eh, em = compare(s, Uh, Um, t_end=0.1)
    assert abs(a[0] - b[0]) <= 1e-3 * a[0]
    err = max(eh.max(), em.max())
    assert err <= TOL_MIXED, (eh, em)


def test_mixed_exponential_collisions(gpu_lib):
    s, Uh, Um = ics.shock_tube_member(600, col=1.0e4, pratio=10.0, dratio=5.0, ion_frac=0.2)
    a, b, eh, em = compare(s, Uh, Um, t_end=0.05)
    err = max(eh.max(), em.max())
    assert err <= TOL_MIXED, (eh, em)


@pytest.mark.parametrize("bnd", [[2, 2, 10, 10], [10, 10, 2, 2], [3, 4, 5, 6]])
def test_mixed_mirror_walls(gpu_lib, bnd):
    """Mirror faces: the FP32 HLL averages of vn and Bn must cancel to exactly zero there, as
    in FP64, or the wall's tangential fluxes take the other side's sign."""
    s, Uh, Um = ics.orszag_tang(48, flag_bnd=bnd + [1, 1], flag_divb=0)
    a, b, eh, em = compare(s, Uh, Um, nsteps=40)
    assert a[1] == b[1] == 40 and abs(a[0] - b[0]) <= 1e-5 * a[0]
    assert max(eh.max(), em.max()) <= TOL_MIXED, (eh, em)


def test_mixed_roundtrip_upload_download(gpu_lib):
    """upload splits FP64 into (hi, lo) and download joins it back to ~2^-48."""
    s, Uh, Um = ics.orszag_tang(40, precision=PIP_MIXED)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        h, m = c.download()
    np.testing.assert_allclose(h, Uh, rtol=1e-13, atol=1e-300)
    np.testing.assert_allclose(m, Um, rtol=1e-13, atol=1e-300)


def test_paired_solvers_match_scalar(tmp_path):
    """The mixed form's FP32 HLLD/HLLC with each face's left and right work in packed FP32x2
    arithmetic (pip_pair.cuh) against the scalar reciprocal forms, over 2^20 seeded faces per
    kind, differences relative to the face's flux scale.  Unrelated random states (kind 0,
    with supersonic faces) carry the FP32 cancellation of the energy flux between branches;
    nearby states, mirror pairs and near-zero Bn stay at rounding."""
    import os
    import re
    import subprocess
    from pip_b200 import build as b
    here = os.path.dirname(os.path.abspath(__file__))
    exe = tmp_path / "pair_flux_check"
    subprocess.run([b.nvcc()] + b.ARCH + ["-O3", "-std=c++17", "--expt-relaxed-constexpr",
                    "-ftz=true", "-prec-div=false", "-prec-sqrt=false",
                    os.path.join(here, "pair_flux_check.cu"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    print(out)
    kinds = {int(m.group(1)): (float(m.group(2)), float(m.group(3)))
             for m in re.finditer(r"kind (\d) faces \d+ hlld_max (\S+) hllc_max (\S+)", out)}
    assert sorted(kinds) == [0, 1, 2, 3]
    assert max(kinds[0]) <= 1e-3
    for k in (1, 2, 3):
        assert max(kinds[k]) <= 1e-5, (k, kinds[k])
    side = re.search(r"supersonic_left (\d+) supersonic_right (\d+) subsonic (\d+)", out)
    assert all(int(x) > 0 for x in side.groups())
    assert re.search(r"nonfinite 0", out)

