"""Discrete adjoint of the FP64 run (include/pip_adjoint.h, pip_b200.adjoint) on the GPU.

* its forward is the FP64 time loop of pip_run, bit for bit;
* its gradient equals the torch.autograd gradient of an independent FP64 restatement of the
  same discrete run (tests/torch_pip2d.py) on small grids, including a run whose dt is set
  by the collision bound;
* its gradient with respect to the initial perturbation field and alpha_c matches central
  finite differences of the GPU forward (step 1e-6, 16 random directions) for the
  two-fluid linear wave-damping run at 512x256, 500 steps, checkpoints every 25 steps, and
  on small 1D / non-periodic cases.
"""
import numpy as np
import pytest
import torch

import torch_pip2d as T
from oracle import oracle as O
from pip_b200 import capi, ics
from pip_b200.adjoint import AdjointRun, pip_run, wave_damping_state
from pip_b200.ics import velocity_modes

pytestmark = pytest.mark.gpu

H = 1.0e-6            # finite-difference step
N_DIRS = 16


def prologue_state(s, Uh, Um):
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    Uh0, Um0 = o.state()
    o.close()
    return np.concatenate([Um0, Uh0], axis=0)


def perturbation(s, seed, amp=1.0e-4, kmax=8):
    X, Y = ics._grid(s)
    dv = velocity_modes(X, Y, s.end[0] - s.start[0], s.end[1] - s.start[1], seed, amp, kmax)
    return [torch.from_numpy(d).cuda() for d in dv]


def c5_loss(UN, tgt_vy, tgt_rn, m=2):
    """L2 misfit of the final ion vy and neutral density."""
    vy = UN[2, m:-m, m:-m] / UN[0, m:-m, m:-m]
    rn = UN[8, m:-m, m:-m]
    return ((vy - tgt_vy) ** 2).sum() + ((rn - tgt_rn) ** 2).sum()


def test_adjoint_forward_is_pip_run(gpu_lib):
    s, Uh, Um = ics.wave_damping(64, 32, amp=1.0e-2)
    U0 = prologue_state(s, Uh, Um)
    with capi.Context(s) as c:
        c.upload(U0[8:].copy(), U0[:8].copy())
        st, t, n = c.run(nsteps=30)
        h, m = c.download()
    r = AdjointRun(s, 30, checkpoint_every=7)
    UN = r.forward(torch.from_numpy(U0).cuda()).cpu().numpy()
    assert st == 0 and n == 30
    assert np.array_equal(UN, np.concatenate([m, h], axis=0))
    r.close()


@pytest.mark.parametrize("col", [10.0, 300.0])
def test_adjoint_matches_torch_reference_gradient(gpu_lib, col):
    s, Uh, Um = ics.wave_damping(16, 8, amp=3.0e-2, col=col)
    U0 = prologue_state(s, Uh, Um)
    nsteps = 12
    rng = np.random.default_rng(7)
    w = rng.standard_normal(U0.shape)
    _, _, _, dx, dy, _ = s.coordinates()
    # FP64 reference: autograd of the torch restatement on the CPU
    U0c = torch.from_numpy(U0.copy()).requires_grad_(True)
    acc_ = torch.tensor(col, dtype=torch.float64, requires_grad=True)
    UNc, dts = T.run(U0c, acc_, nsteps, s.gm, s.safety, s.ro_lim, s.pr_lim,
                     torch.from_numpy(dx), torch.from_numpy(dy))
    (torch.from_numpy(w) * UNc).sum().backward()
    # the adjoint on the GPU, three checkpoint segments (5, 5, 2 steps)
    r = AdjointRun(s, nsteps, checkpoint_every=5)
    U0g = torch.from_numpy(U0.copy()).cuda().requires_grad_(True)
    acg = torch.tensor(col, dtype=torch.float64, device="cuda", requires_grad=True)
    UNg = pip_run(U0g, acg, r)
    (torch.from_numpy(w).cuda() * UNg).sum().backward()
    np.testing.assert_allclose(r.dt_history(), np.array([float(d) for d in dts]), rtol=1e-12)
    ref = U0c.grad.numpy()
    got = U0g.grad.cpu().numpy()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= 1e-9, err
    assert abs(acg.grad.item() - acc_.grad.item()) <= 1e-9 * abs(acc_.grad.item())
    r.close()


def fd_check(r, make_state, params, loss_of, col, n_dirs=N_DIRS, seed=0):
    """Adjoint gradient of loss(forward(make_state(params), col)) against central differences
    along n_dirs random directions of params and along col; returns the relative errors."""
    gen = torch.Generator(device="cuda").manual_seed(seed)
    ps = [p.detach().clone().requires_grad_(True) for p in params]
    ac = torch.tensor(col, dtype=torch.float64, device="cuda", requires_grad=True)
    L = loss_of(pip_run(make_state(*ps), ac, r))
    L.backward()
    grads = [p.grad.detach() for p in ps]
    gcol = ac.grad.item()

    def L_at(qs, c):
        with torch.no_grad():
            return loss_of(r.forward(make_state(*qs), c)).item()
    errs = []
    for _ in range(n_dirs):
        d = [torch.randn(p.shape, generator=gen, device="cuda", dtype=torch.float64) for p in ps]
        lp = L_at([p.detach() + H * di for p, di in zip(ps, d)], col)
        lm = L_at([p.detach() - H * di for p, di in zip(ps, d)], col)
        fd = (lp - lm) / (2.0 * H)
        an = sum((g * di).sum().item() for g, di in zip(grads, d))
        errs.append(abs(an - fd) / max(abs(fd), 1e-300))
    lp = L_at([p.detach() for p in ps], col + H)
    lm = L_at([p.detach() for p in ps], col - H)
    fd = (lp - lm) / (2.0 * H)
    return np.array(errs), abs(gcol - fd) / max(abs(fd), 1e-300), L.item()


def c5_case(nx, ny, nsteps, K=25):
    s, _, _ = ics.wave_damping(nx, ny, col=10.0)
    st, _, _ = ics.wave_damping(nx, ny, seed=5151, col=20.0)
    r = AdjointRun(s, nsteps, checkpoint_every=K)
    # target: forward run with alpha_c = 20 from the seed-5151 perturbation
    tv = perturbation(st, 5151)
    UT = r.forward(wave_damping_state(st, *tv), 20.0)
    tgt_vy = (UT[2, 2:-2, 2:-2] / UT[0, 2:-2, 2:-2]).clone()
    tgt_rn = UT[8, 2:-2, 2:-2].clone()
    pv = perturbation(s, 5150)
    return s, r, pv, (lambda U: c5_loss(U, tgt_vy, tgt_rn))


def test_adjoint_fd_small_wave_damping(gpu_lib):
    s, r, pv, loss = c5_case(64, 32, 60)
    errs, ecol, L = fd_check(r, lambda a, b: wave_damping_state(s, a, b), pv, loss, 10.0)
    print("fd rel errors", errs.max(), np.median(errs), "col", ecol, "L", L)
    assert L > 0
    assert errs.max() <= 1e-5 and ecol <= 1e-5
    r.close()


def test_adjoint_fd_c5_full_size(gpu_lib):
    """512x256, 500 FP64 steps, checkpoints every 25 steps."""
    s, r, pv, loss = c5_case(512, 256, 500)
    errs, ecol, L = fd_check(r, lambda a, b: wave_damping_state(s, a, b), pv, loss, 10.0)
    print("C5 fd rel errors max %.3e median %.3e col %.3e L %.6e"
          % (errs.max(), np.median(errs), ecol, L))
    print("forward ms %.2f backward ms %.2f" % (r.forward_ms, r.backward_ms))
    assert errs.max() <= 1e-5 and ecol <= 1e-5
    r.close()


def test_adjoint_fd_nonperiodic_2d(gpu_lib):
    """Reflecting x boundaries (sign flips of the normal components), outflow y boundaries."""
    s, Uh, Um = ics.wave_damping(32, 16, amp=1.0e-2, flag_bnd=[2, 2, 10, 10, 1, 1])
    U0 = torch.from_numpy(prologue_state(s, Uh, Um)).cuda()
    r = AdjointRun(s, 40, checkpoint_every=9)
    w = torch.randn(U0.shape, generator=torch.Generator(device="cuda").manual_seed(3),
                    device="cuda", dtype=torch.float64)
    errs, ecol, L = fd_check(r, lambda U: U, [U0], lambda U: (w * U).sum(), 10.0, n_dirs=8)
    print("nonperiodic fd", errs.max(), ecol)
    assert errs.max() <= 1e-5 and ecol <= 1e-5
    r.close()


def test_adjoint_fd_1d(gpu_lib):
    """A smooth 1D two-fluid wave with outflow boundaries."""
    s, Uh, Um = ics.brio_wu(96, col=30.0)
    x = s.coordinates()[0]
    k = 2.0 * np.pi
    ro = 1.0 + 0.1 * np.sin(k * x)
    vx = 0.05 * np.cos(k * x)
    vy = 0.02 * np.sin(2 * k * x)
    pr = 0.6 + 0.05 * np.cos(k * x)
    by = 1.0 + 0.1 * np.sin(k * x)
    zero = np.zeros_like(x)
    Uh = ics.pv2cq_hd(s, 0.5 * ro[None], vx[None], vy[None], zero[None], pr[None] / 3.0)
    Um = ics.pv2cq_mhd(s, 0.5 * ro[None], vx[None], vy[None], zero[None], 2.0 * pr[None] / 3.0,
                       0.75 + zero[None], by[None], zero[None])
    U0 = torch.from_numpy(prologue_state(s, Uh, Um)).cuda()
    r = AdjointRun(s, 50, checkpoint_every=25)
    w = torch.randn(U0.shape, generator=torch.Generator(device="cuda").manual_seed(4),
                    device="cuda", dtype=torch.float64)
    errs, ecol, L = fd_check(r, lambda U: U, [U0], lambda U: (w * U).sum(), 30.0, n_dirs=8)
    print("1d fd", errs.max(), ecol)
    assert errs.max() <= 1e-5 and ecol <= 1e-5
    r.close()


def test_adjoint_rejects_unsupported(gpu_lib):
    s, _, _ = ics.orszag_tang(32)   # flag_divb = 1
    with pytest.raises(capi.PipError):
        AdjointRun(s, 10)
