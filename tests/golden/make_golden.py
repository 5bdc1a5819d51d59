"""Writes the golden fixtures of tests/golden/ from the CPU restatement (oracle/).

Each fixture stores the initial state, the run length and the state after the run for a
small case of a benchmark configuration, so that tests can check the oracle against
itself over time (regressions) and the GPU against stored vectors without the oracle.
Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from pip_b200 import ics  # noqa: E402

# name -> (IC function, positional args, keyword args, steps, t_end)
CASES = {
    "brio_wu_64_s1": ("brio_wu", [64], {}, 1, None),
    "brio_wu_64_s2": ("brio_wu", [64], {}, 2, None),
    "brio_wu_64_s50": ("brio_wu", [64], {}, 50, None),
    "brio_wu_1024_t0.1": ("brio_wu", [1024], {}, 0, 0.1),
    "orszag_tang_16_s1": ("orszag_tang", [16], {}, 1, None),
    "orszag_tang_16_s2": ("orszag_tang", [16], {}, 2, None),
    "orszag_tang_24_s30": ("orszag_tang", [24], {}, 30, None),
    "member_exp_48_s40": ("shock_tube_member", [48], dict(col=2.0e3, pratio=5.0, dratio=3.0,
                                                          ion_frac=0.3), 40, None),
    "kh_ir_32x16_s12": ("kelvin_helmholtz", [32, 16], {}, 12, None),
    "mirror_codes_20_s10": ("orszag_tang", [20], dict(flag_bnd=[3, 4, 5, 6, 1, 1]), 10, None),
}


def make(name):
    fn, args, kw, steps, t_end = CASES[name]
    s, Uh, Um = getattr(ics, fn)(*args, **kw)
    st, t, n, Uh2, Um2, _ = O.run_case(s, Uh, Um, nsteps=steps, t_end=t_end, threads=4)
    assert st == 0
    meta = dict(fn=fn, args=args, kw=kw, steps=int(n), t_end=t_end, time=t)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), U_h0=Uh, U_m0=Um, U_h=Uh2, U_m=Um2,
                        meta=np.array(json.dumps(meta)))


def load(name):
    """(settings, U_h0, U_m0, U_h, U_m, meta) of a fixture."""
    z = np.load(os.path.join(HERE, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    s, _, _ = getattr(ics, meta["fn"])(*meta["args"], **meta["kw"])
    return s, z["U_h0"], z["U_m0"], z["U_h"], z["U_m"], meta


if __name__ == "__main__":
    for name in CASES:
        make(name)
        print("wrote", name)
