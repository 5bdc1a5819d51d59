"""Sensitivity of the Dedner potential psi on the 2D two-fluid Orszag-Tang run.

Runs, in lockstep on one GPU: the plain FP64 path (FMA build) as the reference; the FMA-free
FP64 build (a rounding-only change); the FP64 path from an initial state whose Bx and By
carry white relative noise of 1e-7 or of 1e-10; the FP64 path from the initial state
rounded once to FP32; and the FP32-mixed form.  At each checkpoint it prints the relative
L1 error against the reference of the 13 physical fields (max) and of psi, and writes
psi_probe_N.json (and the final psi differences, psi_fields_N.npz) into --out.

    python tests/psi_sensitivity.py [--n 1024] [--checkpoints 10,100,500,1000,2000] [--out DIR]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

from helpers import interior, rel_l1  # noqa: E402
from pip_b200 import capi, ics  # noqa: E402
from pip_b200.params import PIP_MIXED  # noqa: E402

NAMES = ["ro_p", "mx_p", "my_p", "mz_p", "en_p", "bx", "by", "bz", "psi",
         "ro_n", "mx_n", "my_n", "mz_n", "en_n"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--checkpoints", default="10,100,500,1000,2000")
    ap.add_argument("--out", default=".")
    args = ap.parse_args()
    ck_list = [int(x) for x in args.checkpoints.split(",")]
    s, Uh, Um = ics.orszag_tang(args.n)
    rng = np.random.default_rng(7)

    def pert_b(Um, eps):
        Um = Um.copy()
        for n in (5, 6):
            Um[n] *= 1.0 + eps * rng.uniform(-1, 1, size=Um[n].shape)
        return Um

    f32 = lambda a: a.astype(np.float32).astype(np.float64)
    runs = {
        "fp64": (s, Uh, Um),
        "fp64_fma_free": (s.overrides(fp_exact=1), Uh, Um),
        "fp64_B_noise_1e-7": (s, Uh, pert_b(Um, 1e-7)),
        "fp64_B_noise_1e-10": (s, Uh, pert_b(Um, 1e-10)),
        "fp64_start_rounded_to_fp32": (s, f32(Uh), f32(Um)),
        "mixed": (s.overrides(precision=PIP_MIXED), Uh, Um),
    }
    ctx = {}
    for k, (ss, h, m) in runs.items():
        c = capi.Context(ss)
        c.upload(h, m)
        c.prologue()
        ctx[k] = c
    out = {"n": args.n, "l1": {}}
    done = 0
    t0 = time.time()
    for ck in ck_list:
        st = {}
        for k, c in ctx.items():
            r = c.run(nsteps=ck - done)
            assert r[0] == 0, (k, r)
            h, m = c.download()
            st[k] = (interior(h, s), interior(m, s), r[1])
        done = ck
        ah, am, _ = st["fp64"]
        for k, (h, m, t) in st.items():
            if k == "fp64":
                continue
            e = np.concatenate([rel_l1(m, am), rel_l1(h, ah)])
            rec = {nm: float(v) for nm, v in zip(NAMES, e)}
            rec["t"] = t
            out["l1"].setdefault(k, {})[str(ck)] = rec
        print(ck, {k: "max13 %.2e psi %.2e" % (max(v[str(ck)][n] for n in NAMES if n != "psi"),
                                               v[str(ck)]["psi"])
                   for k, v in out["l1"].items()}, flush=True)
        if ck == ck_list[-1]:
            psi = am[8]
            np.savez_compressed(os.path.join(args.out, "psi_fields_%d.npz" % args.n),
                                psi64=psi.astype(np.float32),
                                dmixed=(st["mixed"][1][8] - psi).astype(np.float32))
    for c in ctx.values():
        c.close()
    out["wall_s"] = time.time() - t0
    with open(os.path.join(args.out, "psi_probe_%d.json" % args.n), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
