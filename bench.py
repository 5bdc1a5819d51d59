#!/usr/bin/env python
"""Benchmark of the PIP two-fluid finite-volume step on B200.

Prints ONE JSON line.  A "step" is one full RK2 time step of the two-fluid solver
(cfl + run_solver + cfl of main.f90) over the whole grid.  The workload is the 2D
two-fluid Orszag-Tang vortex at 1024x1024 (periodic, 90 % neutral by mass,
alpha_c = 1e3, Dedner cleaning, CFL 0.3) with synthetic initial data.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: cell-updates/s = interior cells x steps / device time (CUDA events on the
  library's stream around the device loop, state resident in HBM; the two state arrays
  (2 x 118 MB) exceed the 126 MB L2, so no flush between steps).
* e2e: the same metric through the public C ABI with pinned host buffers:
  pip_upload + pip_run + pip_download, copies inside the timed region.
* roofline: the stage-2 kernel (the heavier of the two per-step kernels) against the
  measured HBM copy bandwidth; algorithmic bytes per cell of that kernel = read U1 and U0,
  write U2 = 3 x 14 x 8 B.
* cpu_baseline: the CPU restatement on all host cores, bounded sample of the same workload.
* --impl reference: the reference's own algorithm on host cores (the reference is Fortran +
  MPI + HDF5 and cannot be built on this image; its CPU restatement runs instead).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "2-fluid cell-updates/s, FP32-mixed vs FP64 at L1<=1e-5; adjoint/forward cost"
UNIT = "cell-updates/s"
N_GRID = 1024
WORKLOAD = ("2D two-fluid Orszag-Tang vortex 1024x1024 (+2 ghosts), periodic, 90% neutral "
            "by mass, alpha_c=1e3, gamma=5/3, Dedner psi, CFL 0.3, minmod-MUSCL + HLLD/HLLC, RK2")
FP64_BYTES_PER_CELL_STEP = 5 * 14 * 8     # stage 1: R U0 + W U1; stage 2: R U1, U0 + W U2
FP64_BYTES_PER_CELL_STAGE2 = 3 * 14 * 8


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(key):
    """DRAM bytes per launch from the committed ncu summary (profiles/ncu_traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            d = json.load(f)
        v = d.get(key)
        return None if v is None else float(v)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.t:
                self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(target_s: float = 15.0, threads: int = 0):
    """The CPU restatement on OT 1024^2 with all host cores for about target_s seconds."""
    from oracle import oracle as O
    from pip_b200 import ics
    threads = threads or os.cpu_count() or 1
    O.set_threads(threads)
    s, Uh, Um = ics.orszag_tang(N_GRID)
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    cells = N_GRID * N_GRID
    t0 = time.perf_counter()
    o.run(nsteps=1)
    t1 = time.perf_counter()
    one = t1 - t0
    extra = max(0, int(target_s / max(one, 1e-3)) - 1)
    steps = 1
    if extra:
        t0 = time.perf_counter()
        o.run(nsteps=extra)
        t1 = time.perf_counter()
        steps = extra
        one = (t1 - t0) / extra
    o.close()
    return {"value": cells / one, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "OT 1024x1024 FP64, %d timed step(s) after 1 untimed, %d OpenMP threads"
                      % (steps, threads), "s_per_step": one}


def run_reference(args):
    """--impl reference: the reference algorithm on host cores (CPU restatement)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    budget = float(os.environ.get("PIP_REF_BUDGET_S", "90"))
    from oracle import oracle as O
    from pip_b200 import ics
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    s, Uh, Um = ics.orszag_tang(N_GRID)
    o = O.Oracle(s, Uh, Um)
    o.prologue()
    t0 = time.perf_counter()
    o.run(nsteps=max(1, min(args.warmup, 1)))
    warm = time.perf_counter() - t0
    steps = max(1, min(args.steps, int(budget / max(warm, 1e-3))))
    t0 = time.perf_counter()
    st, _, n, _ = o.run(nsteps=steps)
    dt = time.perf_counter() - t0
    o.close()
    cells = N_GRID * N_GRID
    val = cells * n / dt
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": n, "warmup": 1, "ms_per_step": 1e3 * dt / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": cells, "precision": "fp64",
                   "parallelism": "host OpenMP, %d threads" % threads},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "%d of the requested %d steps (time budget %.0f s)"
                                   % (n, args.steps, budget)},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference is Fortran+MPI+HDF5 with no compiler on this image; the FP64 CPU "
                "restatement of its algorithm is timed",
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=N_GRID, help="grid size (default 1024)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.warmup < 3:
        args.warmup = 3

    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    torch.cuda.init()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from pip_b200 import build, capi, ics
    build.build()
    n = args.n
    cells = n * n
    s, Uh, Um = ics.orszag_tang(n)

    # ---------------------------------------------------------------- device-resident value
    ctx = capi.Context(s)
    ctx.upload(Uh, Um)
    ctx.prologue()
    ctx.run(nsteps=args.warmup)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        st, t, nstep, ms = ctx.run_timed(nsteps=args.steps)
    torch.cuda.synchronize()
    if st != 0 or nstep != args.steps:
        raise RuntimeError("timed run ended with status %d after %d steps" % (st, nstep))
    ms_max = ms
    if dist:
        tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_max = float(tt.item())
    value = world * cells * args.steps / (ms_max * 1e-3)
    launches = ctx.kernels_per_run(args.steps)

    # ---------------------------------------------------------------- per-kernel roofline
    nk = min(200, args.steps)
    ms1, ms2, msstep = ctx.stage_ms(nk)
    peak, peak_kind = measured_peaks()
    achieved2 = FP64_BYTES_PER_CELL_STAGE2 * cells / (ms2 * 1e-3) / 1e9
    traffic = ncu_traffic("stage2_fp64_ot1024")
    ctx.close()

    # ---------------------------------------------------------------- e2e through the C ABI
    shape_h, shape_m = Uh.shape, Um.shape
    ph = torch.empty(shape_h, dtype=torch.float64, pin_memory=True).numpy()
    pm = torch.empty(shape_m, dtype=torch.float64, pin_memory=True).numpy()
    ph[...] = Uh
    pm[...] = Um
    oh = torch.empty(shape_h, dtype=torch.float64, pin_memory=True).numpy()
    om = torch.empty(shape_m, dtype=torch.float64, pin_memory=True).numpy()
    ctx = capi.Context(s)
    ctx.upload(ph, pm)
    ctx.run(nsteps=args.warmup)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.upload(ph, pm)
    ctx.run(nsteps=args.steps)
    ctx.download(oh, om)
    e2e_s = time.perf_counter() - t0
    ctx.close()
    if dist:
        tt = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    state_bytes = (Uh.nbytes + Um.nbytes)
    e2e = {"value": world * cells * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": state_bytes / args.steps,
           "how": "pip_upload (pinned host) + pip_run(%d steps) + pip_download, wall clock "
                  "around the synchronous C ABI calls" % args.steps}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_sample()
        cpu.pop("s_per_step", None)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": cells, "precision": "fp64 (plain drop-in path)",
                   "l2": "inputs larger than L2 (2 x %.0f MB state arrays vs 126 MB L2)"
                         % (state_bytes / 1e6),
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved2, "peak": peak, "unit": "GB/s",
                     "frac": achieved2 / peak, "traffic": traffic,
                     "kernel": "stage_kernel<2,9,2> (stage 2: fluxes+source+update+2x cfl)",
                     "algorithmic_bytes_per_cell": FP64_BYTES_PER_CELL_STAGE2,
                     "peak_kind": peak_kind, "ms_stage1": ms1, "ms_stage2": ms2,
                     "step_achieved_gbs": FP64_BYTES_PER_CELL_STEP * cells / (msstep * 1e-3) / 1e9},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
