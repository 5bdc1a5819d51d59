"""Batched ensemble of 1D and 2D two-fluid runs (include/pip_ensemble.h) against single runs."""
import numpy as np
import pytest

from helpers import rel_l1
from pip_b200 import capi, ics
from pip_b200.ensemble import Ensemble, shock_tube_ensemble
from pip_b200.params import PIP_FP64, PIP_MIXED

pytestmark = pytest.mark.gpu

T_END = 0.02


def members():
    return shock_tube_ensemble(n_runs=7, seed=11, nx_max=300) + \
        [ics.shock_tube_member(64, col=1.0e4, pratio=20.0, dratio=10.0, ion_frac=0.05)]


def single(s, Uh, Um, precision, nsteps=0, t_end=0.0):
    with capi.Context(s.overrides(precision=precision)) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, t, n = c.run(nsteps=nsteps, t_end=t_end)
        return st, t, n, c.download()


def test_ensemble_matches_single_runs(gpu_lib):
    mem = members()
    with Ensemble(mem) as e:
        e.run(t_end=T_END)
        for r, (s, Uh, Um) in enumerate(mem):
            eh, em, t, n, st = e.member(r)
            assert st == 0 and t >= T_END
            # the single-run mixed form does the same per-cell arithmetic; FMA contraction
            # may differ between the two kernels, so they agree to FP32 rounding
            st1, t1, n1, (h1, m1) = single(s, Uh, Um, PIP_MIXED, nsteps=n)
            assert abs(t1 - t) <= 1e-6 * t
            assert max(rel_l1(eh, h1).max(), rel_l1(em, m1).max()) <= 1e-5
            # the FP64 single run after the same number of steps
            st2, t2, n2, (h2, m2) = single(s, Uh, Um, PIP_FP64, nsteps=n)
            assert abs(t2 - t) <= 1e-5 * t
            assert max(rel_l1(eh, h2).max(), rel_l1(em, m2).max()) <= 1e-5


def test_ensemble_configurations_agree(gpu_lib):
    mem = members()[:4]
    out = []
    for threads, cps in ((128, 1), (256, 2), (1024, 1)):
        with Ensemble(mem) as e:
            e.set_config(threads, cps)
            e.run(t_end=0.01)
            out.append([e.member(r) for r in range(len(mem))])
    # each configuration is its own kernel instance: FMA contraction may differ, so the
    # runs agree to FP32 rounding rather than bit for bit
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert a[3] == b[3] and abs(a[2] - b[2]) <= 1e-6 * a[2]
            assert max(rel_l1(a[0], b[0]).max(), rel_l1(a[1], b[1]).max()) <= 1e-6


def test_autotuner_picks_a_valid_configuration(gpu_lib):
    mem = members()
    with Ensemble(mem) as e:
        threads, cps, ms = e.tune(t_probe=0.002)
        assert threads in (128, 256, 512, 1024) and cps >= 1 and ms > 0
        # tuning restores the state: a run from here equals a run of a fresh ensemble
        e.run(t_end=0.005)
        a = [e.member(r) for r in range(len(mem))]
    with Ensemble(mem) as f:
        f.run(t_end=0.005)
        for r in range(len(mem)):
            b = f.member(r)
            assert a[r][3] == b[3]
            assert rel_l1(a[r][1], b[1]).max() <= 1e-6


# The FP32-mixed form against FP64 on config 4's members, measured over all 512 (bench.py
# "ensemble"): median 1.2e-6 relative L1, 24 members above 1e-5, the worst 4.4e-5 (large
# grids with ion fractions of 0.05-0.15, on the small ion density or momentum).  The
# single-run mixed form gives the same on those members (3-5e-5), so this is the precision
# form's, not the batching's; members are held to the measured level.
TOL_C4 = 1e-4


def test_config4_members_match_their_fp64_single_runs(gpu_lib):
    """Config 4 as stated: members of the seeded 512-run ensemble (seed 4242) to t = 0.1,
    each against its own single-run FP64 solve.  The subset holds the largest grid, the
    stiffest alpha_c, the largest pressure ratio and the smallest ion fraction of the 512,
    plus four more drawn with a fixed seed."""
    from pip_b200.ensemble import fp64_single_run_errors
    spec = ics.ensemble_members(512, 4242)
    pick = {max(range(512), key=lambda r: spec[r]["nx"]),
            max(range(512), key=lambda r: spec[r]["col"]),
            max(range(512), key=lambda r: spec[r]["pratio"]),
            min(range(512), key=lambda r: spec[r]["ion_frac"])}
    pick |= set(int(r) for r in np.random.default_rng(99).choice(512, 4, replace=False))
    pick = sorted(pick)
    mem = [ics.shock_tube_member(**spec[r]) for r in pick]
    with Ensemble(mem) as e:
        e.run(t_end=0.1)
        res = [e.member(r) for r in range(len(mem))]
    for (_, _, t, n, st) in res:
        assert st == 0 and t >= 0.1
    errs = fp64_single_run_errors(mem, res)
    for r, (l1, dt_rel) in zip(pick, errs):
        assert dt_rel <= 1e-5, (r, dt_rel)
        print("member %d nx %d alpha_c %.3g: relative L1 %.2e" % (r, spec[r]["nx"], spec[r]["col"],
                                                                 l1.max()))
        assert l1.max() <= TOL_C4, (r, spec[r], l1)


def test_ensemble_with_2d_members(gpu_lib):
    """1D and 2D members of uneven sizes in one persistent launch: the 2D ones (Dedner
    cleaning or not, periodic, reflecting with ionisation/recombination, a ragged grid) are
    walked tile by tile by one CTA with the single-run mixed kernels' tile step.  Each member
    against a single-run mixed context over the same steps (FP32 rounding apart: the two
    kernels may contract differently) and against FP64 on the physical fields."""
    mem = [ics.orszag_tang(32),
           ics.orszag_tang(8, ix0=24, jx0=40, flag_divb=0),
           ics.kelvin_helmholtz(32, 16),
           ics.shock_tube_member(200, col=50.0, pratio=5.0, dratio=4.0, ion_frac=0.4),
           ics.orszag_tang(48, flag_bnd=[2, 2, 10, 10, 1, 1])]
    with Ensemble(mem) as e:
        e.run(t_end=0.01)
        res = [e.member(r) for r in range(len(mem))]
    for (s, Uh, Um), (eh, em, t, n, st) in zip(mem, res):
        assert st == 0 and t >= 0.01 and n >= 2
        st1, t1, n1, (h1, m1) = single(s, Uh, Um, PIP_MIXED, nsteps=n)
        assert abs(t1 - t) <= 1e-6 * t
        assert max(rel_l1(eh, h1).max(), rel_l1(em[:8], m1[:8]).max()) <= 1e-5
        # psi answers FP32 rounding of B a thousand-fold and more (psi ~ 1e-4 |B|): measured
        # 2.4e-5 on the periodic 32^2 member; held to 1e-3
        if em.shape[0] == 9:
            assert rel_l1(em[8:], m1[8:]).max() <= 1e-3
        st2, t2, n2, (h2, m2) = single(s, Uh, Um, PIP_FP64, nsteps=n)
        assert abs(t2 - t) <= 1e-5 * t
        # against FP64 the ensemble is as close as the single-run mixed form is: the
        # precision form's own error (1e-4 on the Kelvin-Helmholtz member's small transverse
        # fields, below 1e-5 elsewhere), not the batching's
        physical = max(rel_l1(eh, h2).max(), rel_l1(em[:8], m2[:8]).max())
        physical1 = max(rel_l1(h1, h2).max(), rel_l1(m1[:8], m2[:8]).max())
        assert physical <= 1.1 * physical1 + 1e-6, (s.ndim, s.ix0, s.jx0, physical, physical1)
        assert physical <= 3e-4, (s.ndim, s.ix0, s.jx0, physical)


def test_2d_members_need_256_threads(gpu_lib):
    mem = [ics.orszag_tang(16)]
    with Ensemble(mem) as e:
        assert capi.lib().pip_ensemble_set_config(e.h, 128, 1) == capi.PIP_ERR_PARAM
        threads, cps, _ = e.tune(t_probe=0.001)
        assert threads >= 256


def test_load_balance_record(gpu_lib):
    mem = members()
    with Ensemble(mem) as e:
        e.set_config(256, 1)
        e.run(t_end=0.005)
        lb = e.load_balance()
    assert lb["slots"] > 0 and 0.0 < lb["busy_fraction"] <= 1.0 + 1e-9
    assert lb["makespan_us"] >= lb["longest_run_us"] > 0.0
    assert lb["makespan_over_ideal"] >= 1.0 - 1e-9


@pytest.mark.parametrize("threads", [512, 256])
def test_cluster_shared_runs_match_one_block(gpu_lib, threads):
    """Runs shared by a thread-block cluster (each block a contiguous part of the cells, the
    cluster barrier between stages, dt reduced over the cluster) evolve as on one block: the
    cells' arithmetic and the exact min/max reductions do not depend on the split, so times
    and step counts are equal; the states agree to the FMA contraction each kernel instance
    gets (measured 1e-14 on 5 of 10^4 values; a stale neighbour cell would show at 1e-3)."""
    mem = [ics.shock_tube_member(3000, col=30.0, pratio=6.0, dratio=3.0, ion_frac=0.3),
           ics.shock_tube_member(2000, col=2.0e3, pratio=12.0, dratio=5.0, ion_frac=0.1),
           ics.shock_tube_member(700, col=1.0, pratio=4.0, dratio=2.0, ion_frac=0.6)] + \
        shock_tube_ensemble(n_runs=5, seed=3, nx_max=400)
    out = {}
    for cl in (1, 4, 8):
        with Ensemble(mem) as e:
            e.set_config(threads, 1)
            e.set_cluster(cl)
            e.run(t_end=0.01)
            plan = e.plan()
            out[cl] = [e.member(r) for r in range(len(mem))]
            lb = e.load_balance()
        if cl == 1:
            assert plan["cluster"] == 1 and plan["shared_runs"] == 0
        else:
            # a handful of runs against >100 slots: every run is above half an even share
            assert plan["cluster"] == cl and plan["shared_runs"] == len(mem)
            assert lb["shared_runs"] == len(mem)
    for cl in (4, 8):
        for a, b in zip(out[1], out[cl]):
            assert a[4] == b[4] == 0 and a[3] == b[3] and a[2] == b[2]
            assert max(rel_l1(a[0], b[0]).max(), rel_l1(a[1], b[1]).max()) <= 1e-12


def test_cluster_rules(gpu_lib):
    with Ensemble([ics.orszag_tang(16)]) as e:
        with pytest.raises(capi.PipError):
            e.set_cluster(4)                        # a 2D run: one block per run
    with Ensemble(members()[:3]) as e:
        e.set_config(1024, 1)
        with pytest.raises(capi.PipError):
            e.set_cluster(4)
        e.set_config(512, 1)
        with pytest.raises(capi.PipError):
            e.set_cluster(3)
        e.set_cluster(0)
        e.run(t_end=0.002)
        assert e.plan()["cluster"] in (4, 8)          # three runs on a whole GPU: shared

