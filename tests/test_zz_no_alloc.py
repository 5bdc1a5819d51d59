"""pip_step_noalloc, the allocation-free run_solver, against pip_step.

Some hosts of this library cannot call cudaMalloc: their device memory belongs to another
layer (an OpenACC or CUDA Fortran data region around the Fortran arrays, or an
application memory pool), or their stepping path must not allocate.  pip_step_noalloc
serves them: it takes a device state the caller already holds and keeps its own scratch
(the stage buffer, the control block, the grid widths) in a fixed-size device array built
into the library.  These tests hold the state in a torch tensor (the test may allocate;
the entry point does not) and check, through the C ABI, that two calls in a row give what
the context-based pip_step gives from the same states.  Both run the same FP64 kernels on
the same inputs, so the results must be equal bit for bit.  The settings the entry point
does not serve are rejected before any GPU work.
This file is collected last, so that a first-failure run has executed every other test.
"""
import ctypes

import numpy as np
import pytest

from pip_b200 import capi, ics
from pip_b200.params import PIP_IR_JEFFERY, PIP_IR_POPESCU, PIP_IR_POPESCU_EQ, PIP_MIXED

pytestmark = pytest.mark.gpu


def two_steps(s, Uh, Um, stream=None):
    """Two pip_step calls and two pip_step_noalloc calls from the same states."""
    import torch
    L = capi.lib()
    params, keep = s.to_params()
    nvm = s.nvar_m
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        for _ in range(2):
            dt, cmax = c.cfl()
            h0, m0 = c.download()
            c.run_solver(dt)
            h1, m1 = c.download()
            U = torch.from_numpy(np.concatenate([m0, h0])).cuda()
            torch.cuda.synchronize()
            if stream is None:
                st = L.pip_step_noalloc(ctypes.byref(params), ctypes.c_void_p(U.data_ptr()),
                                        dt, cmax, None)
                torch.cuda.synchronize()
            else:
                st = L.pip_step_noalloc(ctypes.byref(params), ctypes.c_void_p(U.data_ptr()),
                                        dt, cmax, ctypes.c_void_p(stream.cuda_stream))
                stream.synchronize()
            assert st == capi.PIP_OK, capi.strerror(st)
            out = U.cpu().numpy()
            assert np.array_equal(out[:nvm], m1)
            assert np.array_equal(out[nvm:], h1)


@pytest.mark.parametrize("exact", [0, 1])
def test_step_noalloc_matches_pip_step(gpu_lib, exact):
    s, Uh, Um = ics.orszag_tang(96, fp_exact=exact)
    two_steps(s, Uh, Um)


def test_step_noalloc_1d_brio_wu(gpu_lib):
    """1D, eight ion planes (no Dedner potential), outflow ends."""
    s, Uh, Um = ics.brio_wu(1024)
    two_steps(s, Uh, Um)


def test_step_noalloc_on_a_side_stream(gpu_lib):
    import torch
    side = torch.cuda.Stream()
    s, Uh, Um = ics.orszag_tang(64)
    two_steps(s, Uh, Um, stream=side)


def test_step_noalloc_rejects_oversized_grids(gpu_lib):
    L = capi.lib()
    s, Uh, Um = ics.orszag_tang(600)   # 604*604 cells > PIP_NOALLOC_MAX_CELLS
    params, keep = s.to_params()
    st = L.pip_step_noalloc(ctypes.byref(params), ctypes.c_void_p(1 << 20), 1e-4, 1.0, None)
    assert st == capi.PIP_ERR_PARAM


IR_NORM = dict(t_norm=1.5e4, n_norm=1.0e11, t_ir=10.0)
UNSERVED = {
    "mixed precision": dict(precision=PIP_MIXED),
    "implicit conduction": dict(flag_heat=1, kapper=0.01),
    "alpha_c per cell": dict(flag_col=4),
    "resistivity": dict(flag_resi=1, eta_0=1.0e-4),
    "set_IR type 1": dict(flag_ir=PIP_IR_JEFFERY, **IR_NORM),
    "set_IR type 2": dict(flag_ir=PIP_IR_POPESCU, **IR_NORM),
    "set_IR type 3": dict(flag_ir=PIP_IR_POPESCU_EQ, **IR_NORM),
}


@pytest.mark.parametrize("name", sorted(UNSERVED))
def test_step_noalloc_rejects_unserved_settings(gpu_lib, name):
    """Each of these needs a context's buffers or the mixed kernels; the call returns
    PIP_ERR_PARAM before it touches the GPU (the state pointer is never dereferenced)."""
    L = capi.lib()
    s, Uh, Um = ics.orszag_tang(32)
    s = s.overrides(**UNSERVED[name])
    params, keep = s.to_params()
    st = L.pip_step_noalloc(ctypes.byref(params), ctypes.c_void_p(1 << 20), 1e-4, 1.0, None)
    assert st == capi.PIP_ERR_PARAM, capi.strerror(st)
