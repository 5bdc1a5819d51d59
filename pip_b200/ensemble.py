"""Batched ensembles of independent 1D and 2D two-fluid runs (include/pip_ensemble.h)."""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import capi, ics
from .params import PIP_MIXED, PipParams, Settings


class Ensemble:
    """Many 1D and 2D runs advanced together by one persistent launch (FP32-mixed form)."""

    def __init__(self, members: Sequence[Tuple[Settings, np.ndarray, np.ndarray]]):
        self.settings = [s.overrides(precision=PIP_MIXED) for s, _, _ in members]
        arr = (PipParams * len(members))()
        self._keep = []
        for r, s in enumerate(self.settings):
            p, keep = s.to_params()
            arr[r] = p
            self._keep.append(keep)
        self._arr = arr
        h = ctypes.c_void_p()
        capi._check(capi.lib().pip_ensemble_create(arr, len(members), ctypes.byref(h)),
                    "pip_ensemble_create")
        self.h = h
        self.n = len(members)
        self.shapes = [(U_h.shape, U_m.shape) for _, U_h, U_m in members]
        for r, (_, U_h, U_m) in enumerate(members):
            self.upload(r, U_h, U_m)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            capi.lib().pip_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, r: int, U_h: np.ndarray, U_m: np.ndarray) -> None:
        U_h = np.ascontiguousarray(U_h, dtype=np.float64)
        U_m = np.ascontiguousarray(U_m, dtype=np.float64)
        capi._check(capi.lib().pip_ensemble_upload(self.h, r, capi._ptr(U_h), capi._ptr(U_m)),
                    "pip_ensemble_upload")

    def run(self, t_end: float = 0.0, max_steps: int = 0) -> float:
        """Advance every run; returns the device time of the launch in ms."""
        ms = ctypes.c_float()
        capi._check(capi.lib().pip_ensemble_run(self.h, float(t_end), int(max_steps), ctypes.byref(ms)),
                    "pip_ensemble_run")
        return ms.value

    def member(self, r: int, state: bool = True):
        """(U_h, U_m, time, steps, status) of run r."""
        t = ctypes.c_double()
        n = ctypes.c_int64()
        st = ctypes.c_int()
        if state:
            sh, sm = self.shapes[r]
            U_h, U_m = np.empty(sh), np.empty(sm)
            ph, pm = capi._ptr(U_h), capi._ptr(U_m)
        else:
            U_h = U_m = None
            ph = pm = None
        capi._check(capi.lib().pip_ensemble_member(self.h, r, ph, pm, ctypes.byref(t),
                                                   ctypes.byref(n), ctypes.byref(st)),
                    "pip_ensemble_member")
        return U_h, U_m, t.value, n.value, st.value

    def set_config(self, threads: int, ctas_per_sm: int) -> None:
        capi._check(capi.lib().pip_ensemble_set_config(self.h, int(threads), int(ctas_per_sm)),
                    "pip_ensemble_set_config")

    def set_cluster(self, cluster: int, share: float = 0.25) -> None:
        """Cluster sharing of long runs: 0 chosen per launch, 1 off, 4 or 8 blocks; runs
        whose work exceeds `share` times an even share are shared."""
        capi._check(capi.lib().pip_ensemble_set_cluster(self.h, int(cluster), float(share)),
                    "pip_ensemble_set_cluster")

    def plan(self) -> dict:
        """The last launch's plan: cluster size (1: none), runs shared, blocks launched."""
        c, nb, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        capi._check(capi.lib().pip_ensemble_plan(self.h, ctypes.byref(c), ctypes.byref(nb),
                                                 ctypes.byref(g)), "pip_ensemble_plan")
        return {"cluster": c.value, "shared_runs": nb.value, "grid": g.value}

    def load_balance(self) -> dict:
        """Makespan of the last launch against perfect balance: each run's busy span (device
        timer) from pip_ensemble_timings times the blocks that stepped it; busy fraction =
        sum of block-spans / (slots x makespan).  A run on one block bounds the makespan
        from below by its span; a shared run by its span too, which it cut by its blocks."""
        n = len(self.shapes)
        t0, t1 = np.empty(n), np.empty(n)
        capi._check(capi.lib().pip_ensemble_timings(self.h, capi._ptr(t0), capi._ptr(t1)),
                    "pip_ensemble_timings")
        slots = ctypes.c_int()
        capi._check(capi.lib().pip_ensemble_slots(self.h, ctypes.byref(slots)), "pip_ensemble_slots")
        blocks = np.zeros(n, dtype=np.int32)
        capi._check(capi.lib().pip_ensemble_blocks(self.h, blocks.ctypes.data_as(
            ctypes.POINTER(ctypes.c_int))), "pip_ensemble_blocks")
        ran = t1 >= 0
        span = (t1 - t0)[ran]
        makespan = float(t1[ran].max() - t0[ran].min())
        busy = float((span * np.maximum(blocks[ran], 1)).sum())
        ideal = max(busy / slots.value, float(span.max()))
        return {"makespan_us": makespan, "busy_us": busy, "slots": slots.value,
                "busy_fraction": busy / (slots.value * makespan),
                "longest_run_us": float(span.max()),
                "shared_runs": int((blocks[ran] > 1).sum()),
                "ideal_makespan_us": ideal,
                "makespan_over_ideal": makespan / ideal,
                "makespan_over_even_split": makespan / (busy / slots.value)}

    def tune(self, t_probe: float) -> Tuple[int, int, float]:
        """Autotune (threads per block, blocks per SM) on a probe run; returns the choice."""
        th, cp, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        capi._check(capi.lib().pip_ensemble_tune(self.h, float(t_probe), ctypes.byref(th),
                                                 ctypes.byref(cp), ctypes.byref(ms)),
                    "pip_ensemble_tune")
        return th.value, cp.value, ms.value


def shock_tube_ensemble(n_runs: int = 512, seed: int = 4242, nx_max: Optional[int] = None):
    """Members of the seeded 1D shock-tube ensemble (ics.ensemble_members)."""
    out = []
    for m in ics.ensemble_members(n_runs, seed):
        if nx_max is not None:
            m = dict(m, nx=min(m["nx"], nx_max))
        out.append(ics.shock_tube_member(**m))
    return out


def fp64_single_run_errors(members: Sequence[Tuple[Settings, np.ndarray, np.ndarray]],
                           results: Sequence[Tuple[np.ndarray, np.ndarray, float, int, int]],
                           workers: int = 8):
    """Each ensemble member against its own single-run FP64 solve (a context of the plain
    FP64 path, from the same initial state, the same number of steps).

    results[r] is Ensemble.member(r).  Returns one (relative L1 per variable over the
    interior cells, ion planes then neutral planes; |time difference| / time) per member.
    The single runs go to `workers` host threads, each with its own context and stream (the
    C ABI calls release the GIL), so several run on the GPU at once.
    """
    from concurrent.futures import ThreadPoolExecutor

    from .params import PIP_FP64

    def one(r):
        s, U_h, U_m = members[r]
        eh, em, t, n, _ = results[r]
        with capi.Context(s.overrides(precision=PIP_FP64)) as c:
            c.upload(U_h, U_m)
            c.prologue()
            st, t64, n64 = c.run(nsteps=n)
            if st != 0 or n64 != n:
                raise RuntimeError("FP64 single run %d ended with status %d after %d of %d steps"
                                   % (r, st, n64, n))
            h64, m64 = c.download()
        m0 = s.margin[0]
        num = [np.abs(a[:, :, m0:-m0] - b[:, :, m0:-m0]).sum(axis=(1, 2))
               for a, b in ((em, m64), (eh, h64))]
        den = [np.abs(b[:, :, m0:-m0]).sum(axis=(1, 2)) for b in (m64, h64)]
        num, den = np.concatenate(num), np.concatenate(den)
        l1 = np.where(den > 0, num / np.where(den > 0, den, 1.0), num)
        return l1, abs(t - t64) / t64

    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(one, range(len(members))))
