"""Differentiable FP64 two-fluid runs: the discrete adjoint of include/pip_adjoint.h behind a
``torch.autograd.Function``.

``AdjointRun`` owns one ``pip_adj`` handle (device storage for the checkpoints of a run of
``nsteps`` steps).  ``pip_run(U0, col, runner)`` advances a device state through the FP64
time loop of ``pip_run`` (main.f90:31-68) and returns the final state; its backward pulls the
cotangent of the final state back to ``U0`` and to the collision coefficient ``col``
(alpha_c), recomputing each segment of ``checkpoint_every`` steps from its checkpoint.

State tensors are CUDA float64 tensors of shape ``(nvar_m + 5, jx, ix)``: the ion planes
(ro, mx, my, mz, en, bx, by, bz) then the neutral planes (ro, mx, my, mz, en), ghost cells
included -- the planes of the Fortran ``U_m(ix,jx,1,nvar_m)`` and ``U_h(ix,jx,1,5)`` arrays.
There is no CPU path: the library must be built and a GPU present.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np
import torch

from .capi import PipError, PIP_OK, lib
from .params import Settings


def pack_state(U_h, U_m, device="cuda") -> torch.Tensor:
    """(nvar_m + 5, jx, ix) float64 tensor from the Fortran-layout arrays U_h, U_m."""
    U_m = torch.as_tensor(np.asarray(U_m) if not torch.is_tensor(U_m) else U_m, dtype=torch.float64)
    U_h = torch.as_tensor(np.asarray(U_h) if not torch.is_tensor(U_h) else U_h, dtype=torch.float64)
    return torch.cat([U_m, U_h], dim=0).to(device).contiguous()


def unpack_state(U: torch.Tensor, nvar_m: int = 8):
    """(U_h, U_m) views of a packed state."""
    return U[nvar_m:], U[:nvar_m]


class AdjointRun:
    """A ``pip_adj`` handle: forward runs of ``nsteps`` steps with a checkpoint every
    ``checkpoint_every`` steps, and their adjoint."""

    def __init__(self, s: Settings, nsteps: int, checkpoint_every: int = 25):
        if not torch.cuda.is_available():
            raise RuntimeError("AdjointRun needs a CUDA device")
        self.s = s
        self.nsteps = int(nsteps)
        self.K = int(checkpoint_every)
        self.params, self._keep = s.to_params()
        self.col = float(s.col)
        ix, jx, _ = s.shape
        self.shape = (s.nvar_m + 5, jx, ix)
        self.device = torch.device("cuda", torch.cuda.current_device())
        h = ctypes.c_void_p()
        st = lib().pip_adj_create(ctypes.byref(self.params), self.nsteps, self.K, ctypes.byref(h))
        if st != PIP_OK:
            raise PipError(st, "pip_adj_create")
        self.h = h
        self.generation = 0
        self.forward_ms = None
        self.backward_ms = None

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            lib().pip_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_state(self, U: torch.Tensor) -> torch.Tensor:
        if not torch.is_tensor(U) or U.dtype != torch.float64 or U.device.type != "cuda":
            raise TypeError("state must be a CUDA float64 tensor")
        if tuple(U.shape) != self.shape:
            raise ValueError("state shape %s, expected %s" % (tuple(U.shape), self.shape))
        return U.contiguous()

    def forward(self, U0: torch.Tensor, col: Optional[float] = None) -> torch.Tensor:
        """Final state after ``nsteps`` steps from ``U0`` (not modified)."""
        U0 = self._check_state(U0)
        if col is not None and float(col) != self.col:
            st = lib().pip_adj_set_col(self.h, float(col))
            if st != PIP_OK:
                raise PipError(st, "pip_adj_set_col")
            self.col = float(col)
        out = torch.empty_like(U0)
        ms = ctypes.c_float()
        torch.cuda.current_stream().synchronize()
        st = lib().pip_adj_forward(self.h, ctypes.c_void_p(U0.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), self.nsteps, ctypes.byref(ms))
        if st != PIP_OK:
            raise PipError(st, "pip_adj_forward")
        self.forward_ms = ms.value
        self.generation += 1
        return out

    def backward(self, gN: torch.Tensor) -> Tuple[torch.Tensor, float]:
        """(dL/dU0, dL/dcol) for the cotangent gN = dL/dUN of the last forward run."""
        gN = self._check_state(gN)
        g0 = torch.empty_like(gN)
        gc = ctypes.c_double()
        ms = ctypes.c_float()
        torch.cuda.current_stream().synchronize()
        st = lib().pip_adj_backward(self.h, ctypes.c_void_p(gN.data_ptr()),
                                    ctypes.c_void_p(g0.data_ptr()), ctypes.byref(gc), ctypes.byref(ms))
        if st != PIP_OK:
            raise PipError(st, "pip_adj_backward")
        self.backward_ms = ms.value
        return g0, gc.value

    def stage_vjp(self, stage: int, Us: torch.Tensor, lam: torch.Tensor, dt: float):
        """Unit-level reverse of one RK stage: (cotangent of Us, dt_sub <lam, dU/d dt_sub>,
        <lam, dU/dalpha_c>) for the cotangent lam of the stage output (interior cells)."""
        Us = self._check_state(Us)
        lam = self._check_state(lam)
        out = torch.empty_like(Us)
        dot = ctypes.c_double()
        dcol = ctypes.c_double()
        torch.cuda.current_stream().synchronize()
        st = lib().pip_adj_stage_vjp(self.h, int(stage), ctypes.c_void_p(Us.data_ptr()),
                                     ctypes.c_void_p(lam.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     float(dt), ctypes.byref(dot), ctypes.byref(dcol))
        if st != PIP_OK:
            raise PipError(st, "pip_adj_stage_vjp")
        return out, dot.value, dcol.value

    def fold(self, lam: torch.Tensor) -> torch.Tensor:
        """Adjoint of the ghost fill (a copy of lam with ghost cotangents added to their
        interior sources; ghost entries left as they were)."""
        lam = self._check_state(lam).clone()
        torch.cuda.current_stream().synchronize()
        st = lib().pip_adj_fold(self.h, ctypes.c_void_p(lam.data_ptr()))
        if st != PIP_OK:
            raise PipError(st, "pip_adj_fold")
        return lam

    def dt_history(self) -> np.ndarray:
        n = ctypes.c_int64()
        out = np.empty(self.nsteps)
        st = lib().pip_adj_dt(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              self.nsteps, ctypes.byref(n))
        if st != PIP_OK:
            raise PipError(st, "pip_adj_dt")
        return out[: n.value]


class _PipRun(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, col, runner):
        UN = runner.forward(U0.detach(), float(col))
        ctx.runner = runner
        ctx.generation = runner.generation
        ctx.col_shape = col.shape if torch.is_tensor(col) else None
        ctx.col_dtype = col.dtype if torch.is_tensor(col) else torch.float64
        ctx.col_device = col.device if torch.is_tensor(col) else U0.device
        return UN

    @staticmethod
    def backward(ctx, gN):
        runner = ctx.runner
        if runner.generation != ctx.generation:
            raise RuntimeError("the AdjointRun was run forward again before this backward; "
                               "its checkpoints belong to the later run")
        g0, gc = runner.backward(gN)
        gcol = None
        if ctx.col_shape is not None:
            gcol = torch.full(ctx.col_shape, gc, dtype=ctx.col_dtype, device=ctx.col_device)
        return g0, gcol, None


def pip_run(U0: torch.Tensor, col, runner: AdjointRun) -> torch.Tensor:
    """Differentiable FP64 run of ``runner.nsteps`` steps from ``U0`` with alpha_c = ``col``
    (a float or a scalar tensor that may require grad)."""
    return _PipRun.apply(U0, col, runner)


def wave_damping_state(s: Settings, dvx: torch.Tensor, dvy: torch.Tensor) -> torch.Tensor:
    """Packed initial state of the two-fluid linear wave-damping case (``ics.wave_damping``:
    rho = 1 split by n_fraction, p = 0.6 split by the electron convention, B0 = 1 along x)
    with velocity perturbation fields dvx, dvy of shape (jx, ix) given to both species;
    differentiable in dvx, dvy.  Same operations as ics.pv2cq_hd / pv2cq_mhd."""
    from .ics import fractions
    gm = s.gm
    f_n, f_p, f_p_n, f_p_p = fractions(s.n_fraction)
    zero = torch.zeros_like(dvx)
    one = torch.ones_like(dvx)

    def cons(de, vx, vy, pr, bx):
        vz = zero
        e = pr / (gm - 1.0) + 0.5 * de * (vx * vx + vy * vy + vz * vz)
        planes = [de, de * vx, de * vy, de * vz]
        if bx is None:
            return planes + [e]
        return planes + [e + 0.5 * (bx * bx + zero * zero + zero * zero), bx, zero, zero]
    um = cons(f_p * one, dvx, dvy, f_p_p * 0.6 * one, one)
    uh = cons(f_n * one, dvx, dvy, f_p_n * 0.6 * one, None)
    return torch.stack(um + uh).contiguous()
