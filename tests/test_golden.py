"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py): stored
initial states and the states after a number of steps or to a time, for small cases of
the benchmark configurations.  The oracle must reproduce them bit for bit; the GPU's
FMA-free build must too, except where exp() enters (libm vs CUDA ulps), held to 1e-10."""
import os
import sys

import numpy as np
import pytest

from helpers import rel_l1

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

NAMES = sorted(G.CASES)
EXP_CASES = {"member_exp_48_s40", "kh_ir_32x16_s12"}


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(name):
    from oracle import oracle as O
    s, Uh0, Um0, Uh, Um, meta = G.load(name)
    st, t, n, Uh2, Um2, _ = O.run_case(s, Uh0, Um0, nsteps=meta["steps"] if meta["t_end"] is None else 0,
                                       t_end=meta["t_end"], threads=4)
    assert st == 0 and n == meta["steps"] and t == meta["time"]
    np.testing.assert_array_equal(Uh2, Uh)
    np.testing.assert_array_equal(Um2, Um)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_reproduces_fixture(gpu_lib, name):
    from pip_b200 import capi
    s, Uh0, Um0, Uh, Um, meta = G.load(name)
    s = s.overrides(fp_exact=1)
    with capi.Context(s) as c:
        c.upload(Uh0, Um0)
        c.prologue()
        if meta["t_end"] is None:
            st, t, n = c.run(nsteps=meta["steps"])
        else:
            st, t, n = c.run(t_end=meta["t_end"])
        gh, gm = c.download()
    assert st == 0 and n == meta["steps"]
    if name in EXP_CASES:
        assert max(rel_l1(gh, Uh).max(), rel_l1(gm, Um).max()) <= 1e-10
    else:
        assert t == meta["time"]
        np.testing.assert_array_equal(gh, Uh)
        np.testing.assert_array_equal(gm, Um)
