"""The torch restatement of the 2D step (tests/torch_pip2d.py, the FP64 reference gradient of
the adjoint tests) reproduces the C oracle's trajectory, so that its autograd gradient is
the gradient of the same discrete run.  CPU only."""
import numpy as np
import pytest
import torch

import torch_pip2d as T
from generic_state import generic_state
from oracle import oracle as O
from pip_b200 import ics


def prologue_state(s, Uh, Um):
    """The state after the prologue's cfl rewrite and ghost fill (Initial_rot.f90:152-160)."""
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    Uh0, Um0 = o.state()
    return o, Uh0, Um0


CASES = {
    "periodic": dict(col=10.0),
    "collision_dt": dict(col=300.0),
    "reflect_outflow": dict(col=10.0, flag_bnd=[2, 2, 10, 10, 1, 1]),
    "outflow_reflect": dict(col=10.0, flag_bnd=[10, 10, 2, 2, 1, 1]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_torch_restatement_matches_oracle(case):
    s, _, _ = ics.wave_damping(16, 8, **CASES[case])
    Uh, Um = generic_state(s, 3)
    o, Uh0, Um0 = prologue_state(s, Uh, Um)
    U0 = torch.from_numpy(np.concatenate([Um0, Uh0], axis=0))
    with torch.no_grad():
        UN, dts = T.run(U0, CASES[case]["col"], 12, T.Geom(s))
    st, t, n, hist = o.run(nsteps=12, max_hist=12)
    o_h, o_m = o.state()
    o.close()
    assert st == 0 and n == 12
    np.testing.assert_allclose(np.array([float(d) for d in dts]), hist, rtol=1e-13, atol=0)
    ref = np.concatenate([o_m, o_h], axis=0)
    got = UN.numpy()
    for v in range(13):
        den = np.abs(ref[v, 2:-2, 2:-2]).sum()
        err = np.abs(got[v, 2:-2, 2:-2] - ref[v, 2:-2, 2:-2]).sum()
        assert err <= 1e-12 * max(den, 1e-300) or err < 1e-15 * got[v].size, (v, err, den)


def test_torch_restatement_matches_oracle_1d():
    s, _, _ = ics.brio_wu(48, col=30.0)
    Uh, Um = generic_state(s, 4)
    o, Uh0, Um0 = prologue_state(s, Uh, Um)
    U0 = torch.from_numpy(np.concatenate([Um0, Uh0], axis=0))
    with torch.no_grad():
        UN, dts = T.run(U0, 30.0, 10, T.Geom(s))
    st, t, n, hist = o.run(nsteps=10, max_hist=10)
    o_h, o_m = o.state()
    o.close()
    np.testing.assert_allclose(np.array([float(d) for d in dts]), hist, rtol=1e-13, atol=0)
    ref = np.concatenate([o_m, o_h], axis=0)
    np.testing.assert_allclose(UN.numpy(), ref, rtol=1e-11, atol=1e-14)


def test_torch_restatement_gradient_is_finite_and_nonzero():
    s, Uh, Um = ics.wave_damping(16, 8, amp=3.0e-2)
    _, Uh0, Um0 = prologue_state(s, Uh, Um)
    U0 = torch.from_numpy(np.concatenate([Um0, Uh0], axis=0)).requires_grad_(True)
    ac = torch.tensor(10.0, dtype=torch.float64, requires_grad=True)
    UN, _ = T.run(U0, ac, 4, T.Geom(s))
    loss = (UN[2, 2:-2, 2:-2] ** 2).sum() + (UN[8, 2:-2, 2:-2] ** 2).sum()
    loss.backward()
    assert torch.isfinite(U0.grad).all() and torch.isfinite(ac.grad)
    assert U0.grad.abs().max() > 0 and ac.grad.abs() > 0
