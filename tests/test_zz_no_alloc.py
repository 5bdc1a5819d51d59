"""pip_step_noalloc, the allocation-free run_solver, against pip_step.

Some hosts of this library cannot call cudaMalloc: their device memory belongs to another
layer (an OpenACC or CUDA Fortran data region around the Fortran arrays, or an
application memory pool), or their stepping path must not allocate.  pip_step_noalloc
serves them: it takes a device state the caller already holds and keeps its own scratch
(the stage buffer, the control block, the grid widths) in a fixed-size device array built
into the library.  This test holds the state in a torch tensor (the test may allocate; the
entry point does not) and checks, through the C ABI, that two calls in a row give what
the context-based pip_step gives from the same states, within the FP64 parity tolerance.
It lives in its own file so that a first-failure run has executed every other test first.
"""
import ctypes

import numpy as np
import pytest

from helpers import rel_l1
from pip_b200 import capi, ics

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10


@pytest.mark.parametrize("exact", [0, 1])
def test_step_noalloc_matches_pip_step(gpu_lib, exact):
    import torch
    L = capi.lib()
    s, Uh, Um = ics.orszag_tang(96, fp_exact=exact)
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
            st = L.pip_step_noalloc(ctypes.byref(params), ctypes.c_void_p(U.data_ptr()),
                                    dt, cmax, None)
            assert st == capi.PIP_OK, capi.strerror(st)
            torch.cuda.synchronize()
            out = U.cpu().numpy()
            assert rel_l1(out[:nvm], m1).max() <= TOL_FP64
            assert rel_l1(out[nvm:], h1).max() <= TOL_FP64


def test_step_noalloc_rejects_oversized_grids(gpu_lib):
    L = capi.lib()
    s, Uh, Um = ics.orszag_tang(600)   # 604*604 cells > PIP_NOALLOC_MAX_CELLS
    params, keep = s.to_params()
    st = L.pip_step_noalloc(ctypes.byref(params), ctypes.c_void_p(1 << 20), 1e-4, 1.0, None)
    assert st == capi.PIP_ERR_PARAM
