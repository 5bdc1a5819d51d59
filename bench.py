#!/usr/bin/env python
"""Benchmark of the PIP two-fluid finite-volume step on B200.

Prints ONE JSON line.  A "step" is one full RK2 time step of the two-fluid solver
(cfl + run_solver + cfl of main.f90) over the whole grid.  The workload is the 2D
two-fluid Orszag-Tang vortex at 1024x1024 (periodic, 90 % neutral by mass,
alpha_c = 1e3, Dedner cleaning, CFL 0.3) with synthetic initial data.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: cell-updates/s of the FP32-mixed form = interior cells x steps / device time
  (CUDA events on the library's stream around the device loop, state resident in HBM; the
  state arrays exceed the 126 MB L2, so no flush between steps).  The plain FP64 path is
  timed the same way ("fp64"), and the relative L1 error of the mixed state against the
  FP64 state after the same steps is reported per variable.
* N > 1 GPUs (torchrun, one rank per GPU; or --decompose with one GPU): the y-slab domain
  decomposition of pip_b200.decomp, weak-scaled -- the Orszag-Tang pattern repeated in y
  over [0,1] x [0,N] with one 1024x1024 slab per GPU, a halo exchange (NCCL point-to-point)
  after each RK stage, the cfl candidates (dt MIN, rho/IR-rate MAX) reduced over ranks on
  the device between steps; device time between CUDA events around the step loop, max over
  ranks; value = N x 1024^2 x steps / time.
* e2e: the same metric through the public C ABI with pinned host buffers:
  pip_upload + pip_run + pip_download, copies inside the timed region.
* roofline: the stage-2 kernel (the heavier of the two per-step kernels) against the
  measured HBM copy bandwidth; algorithmic bytes per cell of that kernel: FP64 read U1 and
  U0, write U2 = 3 x 14 x 8 B; mixed read U1, U0.hi, U0.lo, write U2.hi, U2.lo = 14 x 20 B.
* cpu_baseline: the CPU restatement on all host cores, bounded sample of the same workload.
* --impl reference: the reference's own algorithm on host cores (the reference is Fortran +
  MPI + HDF5 and cannot be built on this image; its CPU restatement runs instead).
* adjoint: the discrete adjoint of the two-fluid linear wave-damping run (512x256, 500 FP64
  steps, checkpoints every 25 steps): device time of the plain FP64 forward (pip_run), of
  the checkpointing forward and of the backward (recomputation included), and their ratios.
* ensemble: 512 seeded 1D two-fluid shock tubes (nx log-uniform in [256, 8192], alpha_c
  log-uniform in [0.1, 1e4]) advanced to t = 0.1 in one persistent launch (FP32-mixed):
  sum over runs of interior cells x steps / device time.
* conduction: the 2048x1024 partially ionised Kelvin-Helmholtz run with ionisation/
  recombination and implicit anisotropic conduction (BiCGstab to 1e-10), 1000 steps, plain
  FP64 and FP32-mixed (FP32 inner solve with FP64 iterative refinement): ms per step,
  iterations per step, solver time and GB/s per iteration, mixed-vs-FP64 L1.
* alpha_c_per_cell, resistivity, ionisation_recombination: the FP64 OT step with
  flag_col=5 (set_collisional col_type 4: alpha_c from both temperatures and the drift,
  recomputed at every RK stage), with flag_resi=1, eta_0=1e-4 (resistive_flux on every
  face; margin 3), and with flag_ir=3 (set_IR type 3, the Popescu rates at every stage),
  500 steps each, and their cost over the plain FP64 step.
* nlevel_hydrogen: the FP64 OT step with set_IR type 4 (the 6-level hydrogen model with the
  ionisation-potential energy term), 200 steps on the host loop, and its cost over the plain
  FP64 step.
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
# mixed: stage 1 R hi + W U1 (4+4 B); stage 2 R U1, hi, lo + W hi, lo (5 x 4 B), per plane
MIXED_BYTES_PER_CELL_STEP = 14 * (8 + 20)
MIXED_BYTES_PER_CELL_STAGE2 = 14 * 20
# FP64 pipe busy time per step of the FP64 stage kernels on OT 1024^2, from an ncu --set full
# capture of both kernels (pipe-active fraction x duration, stage 1 0.4500 x 254.5 us +
# stage 2 0.4217 x 278.5 us): the compute floor of the FP64 path
FP64_PIPE_US_PER_STEP = 0.4500 * 254.5 + 0.4217 * 278.5
L1_NAMES = ["ro_n", "mx_n", "my_n", "mz_n", "en_n", "ro_p", "mx_p", "my_p", "mz_p", "en_p",
            "bx", "by", "bz", "ps"]


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
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "utilization.gpu")

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
        """Median SM clock over the samples taken under load (GPU utilisation >= 50 %; all
        samples if none is), the maximum clock and every throttle reason seen active."""
        sm, busy, mx, reasons = [], [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                f = float(parts[1])
                mx = float(parts[2])
            except ValueError:
                continue
            sm.append(f)
            try:
                if len(parts) > 9 and float(parts[9]) >= 50.0:
                    busy.append(f)
            except ValueError:
                pass
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(busy or sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "samples_under_load": len(busy)}


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


def workload_text(n, world, decomposed):
    """The workload of the bench line: the single-GPU Orszag-Tang run, or its weak-scaled
    decomposition over `world` GPUs."""
    if not decomposed:
        return WORKLOAD
    return ("Orszag-Tang pattern repeated in y: %dx%d cells over [0,1]x[0,%d] (periodic), one "
            "%dx%d y-slab per GPU, halo exchange of 2 ghost rows x 14 planes after each RK "
            "stage (NCCL point-to-point), dt MIN and cmax MAX over ranks; physics as the "
            "1024x1024 run" % (n, n * world, world, n, n))


def run_reference(args):
    """--impl reference: the reference algorithm on host cores (CPU restatement)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
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
    # the same untimed warm-up steps as the GPU arm, then as many of the requested steps as
    # the time budget allows
    warmup = max(1, args.warmup)
    t0 = time.perf_counter()
    o.run(nsteps=warmup)
    warm = (time.perf_counter() - t0) / warmup
    steps = max(1, min(args.steps, int(budget / max(warm, 1e-3))))
    t0 = time.perf_counter()
    st, _, n, _ = o.run(nsteps=steps)
    dt = time.perf_counter() - t0
    o.close()
    cells = N_GRID * N_GRID
    val = cells * n / dt
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": n, "warmup": warmup, "ms_per_step": 1e3 * dt / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_text(N_GRID, world, world > 1 or args.decompose),
                   "cells": cells * world, "precision": "fp64",
                   "parallelism": "host OpenMP, %d threads" % threads,
                   "host_sample": "one %dx%d block on the host cores (the per-cell rate of the "
                                  "workload)" % (N_GRID, N_GRID)},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "%d of the requested %d steps (time budget %.0f s)"
                                   % (n, args.steps, budget)},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference is Fortran+MPI+HDF5 with no compiler on this image; the FP64 CPU "
                "restatement of its algorithm is timed",
    }
    print(json.dumps(line), flush=True)
    return 0


def measure(n, precision, steps, warmup, dist, local, exact=0):
    """Device-resident timing of one precision form on OT n x n: returns timings, the
    state after warmup+steps steps and per-kernel durations.  exact=1: the FP64 kernels
    built without FMA contraction."""
    import torch
    from pip_b200 import capi, ics
    s, Uh, Um = ics.orszag_tang(n, precision=precision, fp_exact=exact)
    ctx = capi.Context(s)
    ctx.upload(Uh, Um)
    ctx.prologue()
    ctx.run(nsteps=warmup)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        st, t, nstep, ms = ctx.run_timed(nsteps=steps)
    torch.cuda.synchronize()
    if st != 0 or nstep != steps:
        raise RuntimeError("timed run ended with status %d after %d steps" % (st, nstep))
    state = ctx.download()
    launches = ctx.kernels_per_run(steps)
    ms1, ms2, msstep = ctx.stage_ms(min(200, steps))
    ctx.close()
    return dict(ms=ms, state=state, launches=launches, clocks=clk.summary(), ms1=ms1, ms2=ms2,
                msstep=msstep, settings=s, U=(Uh, Um))


def measure_decomposed(n, precision, steps, warmup, dist, local, world, rank):
    """Weak-scaled decomposition: the Orszag-Tang pattern repeated in y over [0,1] x
    [0,world], 1024 x (1024*world) cells, one 1024x1024 y-slab per rank (pip_b200.decomp:
    cfl -> MIN/MAX over ranks, stage, halo exchange, stage, halo exchange, cfl).  Device
    time between CUDA events on the current stream around the step loop (every call of the
    loop completes before the next starts), max over ranks by the caller."""
    import torch
    from pip_b200 import decomp, ics
    from pip_b200.params import Settings
    sg = ics.orszag_tang(8, precision=precision)[0].overrides(
        ix0=n, jx0=n * world, end=(1.0, float(world), 1.0))
    b = decomp.block_of(sg, world, rank)
    _, Uh, Um = ics.orszag_tang(n, precision=precision, start=b.settings.start, end=b.settings.end)
    eng = decomp.DeviceBlock(b, Uh, Um, device=local)
    comm = decomp.TorchComm(device=torch.device("cuda", local)) if dist else decomp.LocalComm()
    run = decomp.DecomposedRun([eng], comm, divb=sg.divb == 1)
    # the prologue's cfl and ghost fill (physical faces, then the exchanged ones)
    eng.ctx.cfl()
    eng.ctx.pipbnd()
    run.halo()
    if run.run_device(warmup, overlap=True) != 0:
        raise RuntimeError("decomposed warm-up stopped")
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        st = run.run_device(steps, check_every=0, overlap=True)
        e1.record()
        torch.cuda.synchronize()
    if st != 0:
        raise RuntimeError("decomposed run stopped with status %d" % st)
    ms = e0.elapsed_time(e1)
    state = eng.download()
    s_blk = b.settings
    # per step: 2 stage kernels and, per stage, a pack and an unpack per exchanged face
    # (the cfl is fused into stage 2); one cfl kernel opens the run
    halo_faces = sum(1 for v in b.neighbor if v >= 0)
    launches = 1 + steps * (2 + 2 * 2 * halo_faces)
    run.close()
    # the stage kernels' own durations on an undecomposed block of the same size
    from pip_b200 import capi
    with capi.Context(s_blk) as c:
        c.upload(Uh, Um)
        c.prologue()
        ms1, ms2, msstep = c.stage_ms(min(200, steps))
    return dict(ms=ms, state=state, launches=launches, clocks=clk.summary(), ms1=ms1, ms2=ms2,
                msstep=msstep, settings=s_blk, U=(Uh, Um), world_cells=n * n * world)


def e2e_decomposed(n, precision, steps, warmup, dist, local, world, rank):
    """The decomposed run through the public API from pinned host arrays: pip_upload of the
    rank's block, the decomposed steps, pip_download; wall clock, max over ranks by the
    caller."""
    import torch
    from pip_b200 import decomp, ics
    sg = ics.orszag_tang(8, precision=precision)[0].overrides(
        ix0=n, jx0=n * world, end=(1.0, float(world), 1.0))
    b = decomp.block_of(sg, world, rank)
    _, Uh, Um = ics.orszag_tang(n, precision=precision, start=b.settings.start, end=b.settings.end)
    pin = lambda a: torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
    ph, pm, oh, om = pin(Uh), pin(Um), pin(Uh), pin(Um)
    ph[...] = Uh
    pm[...] = Um
    eng = decomp.DeviceBlock(b, ph, pm, device=local)
    comm = decomp.TorchComm(device=torch.device("cuda", local)) if dist else decomp.LocalComm()
    run = decomp.DecomposedRun([eng], comm, divb=sg.divb == 1)
    run.run_device(warmup, overlap=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    eng.ctx.upload(ph, pm)
    st = run.run_device(steps, check_every=0, overlap=True)
    eng.ctx.download(oh, om)
    e2e_s = time.perf_counter() - t0
    run.close()
    if st != 0:
        raise RuntimeError("decomposed e2e run stopped with status %d" % st)
    return e2e_s, Uh.nbytes + Um.nbytes


def e2e_run(s, Uh, Um, steps, warmup, dist):
    """pip_upload (pinned host) + pip_run + pip_download through the C ABI, wall clock."""
    import torch
    from pip_b200 import capi
    pin = lambda a: torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
    ph, pm, oh, om = pin(Uh), pin(Um), pin(Uh), pin(Um)
    ph[...] = Uh
    pm[...] = Um
    ctx = capi.Context(s)
    ctx.upload(ph, pm)
    ctx.run(nsteps=warmup)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.upload(ph, pm)
    ctx.run(nsteps=steps)
    ctx.download(oh, om)
    e2e_s = time.perf_counter() - t0
    ctx.close()
    return e2e_s, Uh.nbytes + Um.nbytes


def measure_variant(n, steps, ms_plain, what, **overrides):
    """The FP64 step of the OT n x n workload with extra physics (overrides of the
    settings), against the plain FP64 step measured before (ms_plain per step)."""
    import torch
    from pip_b200 import capi, ics
    from pip_b200.params import PIP_FP64
    s, Uh, Um = ics.orszag_tang(n, precision=PIP_FP64, **overrides)
    ctx = capi.Context(s)
    ctx.upload(Uh, Um)
    ctx.prologue()
    ctx.run(nsteps=5)
    torch.cuda.synchronize()
    st, t, nstep, ms = ctx.run_timed(nsteps=steps)
    launches = ctx.kernels_per_run(steps)
    ms1, ms2, _ = ctx.stage_ms(min(200, steps))
    ctx.close()
    if st != 0 or nstep != steps:
        raise RuntimeError("%s run ended with status %d after %d steps" % (what, st, nstep))
    return {"workload": "OT %dx%d FP64, %s" % (n, n, what), "steps": steps,
            "ms_per_step": ms / steps, "value": n * n * steps / (ms * 1e-3), "unit": UNIT,
            "ms_stage1": ms1, "ms_stage2": ms2, "over_plain_fp64": (ms / steps) / ms_plain,
            "gpu_launches": launches}


def measure_nlevel(n, steps, ms_plain):
    """The OT n x n FP64 step with set_IR type 4 (the 6-level hydrogen model: rates before
    every stage and cfl, excitation update after every stage, the cfl terms), stepped by the
    host loop, against the plain FP64 step."""
    import torch
    from pip_b200 import capi, ics
    s, Uh, Um, nex = ics.nlevel_orszag_tang(n, flag_ir_type=0, t_ir=1.0, nlev_deriv=1)
    tab = capi.colexp_table(100000)
    ctx = capi.Context(s)
    ctx.upload(Uh, Um)
    ctx.set_nlevel(tab)
    ctx.set_nexcite(nex)
    ctx.prologue()
    ctx.run(nsteps=3)
    torch.cuda.synchronize()
    st, t, nstep, ms = ctx.run_timed(nsteps=steps)
    ctx.close()
    if st != 0 or nstep != steps:
        raise RuntimeError("6-level run ended with status %d after %d steps" % (st, nstep))
    return {"workload": "OT %dx%d FP64, set_IR type 4 (6-level hydrogen, flag_IR_type 0)" % (n, n),
            "steps": steps, "ms_per_step": ms / steps, "value": n * n * steps / (ms * 1e-3),
            "unit": UNIT, "over_plain_fp64": (ms / steps) / ms_plain,
            # per step: 2 x (rates, stage, excitation update) + 2 x (rates, cfl, cfl terms)
            "gpu_launches": 12 * steps}


def measure_adjoint(nsteps=500, K=25):
    """C5: two-fluid linear wave damping 512x256, alpha_c = 10, loss = L2 misfit of the final
    ion vy and neutral density against a forward run with alpha_c = 20 from another seed."""
    import torch
    from pip_b200 import capi, ics
    from pip_b200.adjoint import AdjointRun, pip_run, wave_damping_state
    s, _, _ = ics.wave_damping(512, 256, col=10.0)
    X, Y = ics._grid(s)

    def pert(seed):
        dv = ics.velocity_modes(X, Y, s.end[0] - s.start[0], s.end[1] - s.start[1], seed, 1.0e-4, 8)
        return [torch.from_numpy(d).cuda() for d in dv]
    r = AdjointRun(s, nsteps, checkpoint_every=K)
    UT = r.forward(wave_damping_state(s, *pert(5151)), 20.0)
    tvy = (UT[2, 2:-2, 2:-2] / UT[0, 2:-2, 2:-2]).clone()
    trn = UT[8, 2:-2, 2:-2].clone()
    U0 = wave_damping_state(s, *pert(5150))
    fwd, bwd = [], []
    for _ in range(3):
        U0g = U0.clone().requires_grad_(True)
        ac = torch.tensor(10.0, dtype=torch.float64, device="cuda", requires_grad=True)
        UN = pip_run(U0g, ac, r)
        loss = (((UN[2, 2:-2, 2:-2] / UN[0, 2:-2, 2:-2]) - tvy) ** 2).sum() + \
            ((UN[8, 2:-2, 2:-2] - trn) ** 2).sum()
        loss.backward()
        fwd.append(r.forward_ms)
        bwd.append(r.backward_ms)
    plain = []
    with capi.Context(s) as c:
        Uc = U0.cpu().numpy()
        for _ in range(3):
            c.upload(Uc[8:].copy(), Uc[:8].copy())
            st, t, n, ms = c.run_timed(nsteps=nsteps)
            plain.append(ms)
    r.close()
    f, b, p0 = min(fwd[1:]), min(bwd[1:]), min(plain[1:])
    return {"workload": "2D two-fluid linear wave damping 512x256 (+2 ghosts), periodic, rho=1 "
                        "(50% ions), p=0.6, B0=1 x, alpha_c=10, velocity modes |k|<=8 amp 1e-4 "
                        "(seed 5150); loss: L2 misfit of final ion vy and neutral density vs "
                        "alpha_c=20, seed 5151",
            "steps": nsteps, "checkpoint_every": K, "dtype": "f64",
            "forward_ms": p0, "checkpointed_forward_ms": f, "backward_ms": b,
            "backward_over_forward": b / p0, "gradient_over_forward": (f + b) / p0,
            "target_backward_over_forward": 4.0, "loss": float(loss.item()),
            "dloss_dcol": float(ac.grad.item()),
            "how": "device time (CUDA events in the library) of pip_run over 500 steps, of "
                   "pip_adj_forward (same kernels + checkpoint copies) and of pip_adj_backward "
                   "(recompute of each 25-step segment + reverse sweep); best of 2 after one warm-up"}


def measure_ensemble(n_runs=512, t_end=0.1):
    from pip_b200.ensemble import Ensemble, fp64_single_run_errors, shock_tube_ensemble
    mem = shock_tube_ensemble(n_runs, 4242)
    with Ensemble(mem) as e:
        threads, ctas, _ = e.tune(t_probe=0.002)
        for r, (s, Uh, Um) in enumerate(mem):
            e.upload(r, Uh, Um)
        ms = e.run(t_end=t_end)
        balance = e.load_balance()
        updates = 0
        bad = 0
        results = []
        for r in range(len(mem)):
            res = e.member(r)
            updates += res[3] * mem[r][0].ix0
            bad += res[4] != 0
            results.append(res)
    # every member against its own single-run FP64 solve (same start, same steps)
    t0 = time.time()
    errs = fp64_single_run_errors(mem, results)
    worst = max(range(len(mem)), key=lambda r: float(errs[r][0].max()))
    l1_all = [float(x[0].max()) for x in errs]
    m = mem[worst][0]
    return {"workload": "%d seeded 1D two-fluid shock tubes, nx log-uniform [256, 8192], "
                        "alpha_c log-uniform [0.1, 1e4], to t=%g, FP32-mixed" % (n_runs, t_end),
            "value": updates / (ms * 1e-3), "unit": UNIT, "device_ms": ms,
            "cell_updates": updates, "runs_failed": bad, "threads": threads,
            "ctas_per_sm": ctas,
            "load_balance": {k: (round(v, 4) if isinstance(v, float) else v)
                             for k, v in balance.items()},
            "vs_fp64_single_runs": {
                "members_checked": len(errs), "max_rel_l1": max(l1_all),
                "median_rel_l1": float(statistics.median(l1_all)),
                "members_above_1e-5": sum(x > 1e-5 for x in l1_all),
                "max_rel_time_diff": max(float(x[1]) for x in errs),
                "worst_member": {"index": worst, "nx": m.ix0, "alpha_c": m.col},
                "check_s": time.time() - t0,
                "how": "each member's 13 fields against a plain FP64 single run (pip_run) from "
                       "the same initial state over the same number of steps; relative L1 "
                       "per variable over the interior cells, max over variables"},
            "how": "one persistent launch (CUDA graph), configuration "
                   "chosen by the autotuner on a t=0.002 probe"}


# C3 BiCGstab iteration (three kernels): algorithmic bytes per interior cell -- 5 face-factor
# planes per matrix application; k1 reads p, Ap, r, r0 and writes p', Ap'; k2 reads r, Ap'
# and writes t; k3 reads x, p', t, b, r0 and writes x', r.
HC_BYTES_PER_CELL_ITER = {"f64": 8 * (3 * 5 + 6 + 3 + 7), "f32": 4 * (3 * 5 + 6 + 3 + 7)}


def measure_conduction(nsteps=1000, kapper=0.01):
    """C3: 2D partially ionised Kelvin-Helmholtz 2048x1024 with ionisation/recombination and
    implicit anisotropic conduction (BiCGstab to 1e-10), plain FP64 and FP32-mixed (FP32
    inner solve, FP64 refinement); the same runs without conduction give the cost of the
    solver alone."""
    from pip_b200 import capi, ics
    from pip_b200.params import PIP_FP64, PIP_MIXED
    out = {}
    states = {}
    for name, prec in (("fp64", PIP_FP64), ("mixed", PIP_MIXED)):
        res = {}
        for heat in (1, 0):
            s, Uh, Um = ics.kelvin_helmholtz(2048, 1024, flag_heat=heat, kapper=kapper,
                                             hc_error=1e-10, hc_max=5000, precision=prec)
            with capi.Context(s) as c:
                c.upload(Uh, Um)
                c.prologue()
                st, t, n, ms = c.run_timed(nsteps=nsteps)
                if st != 0 or n != nsteps:
                    raise RuntimeError("C3 %s run ended with status %d after %d steps" % (name, st, n))
                it = c.conduction_iterations if heat else 0
                if heat:
                    states[name] = c.download()
            res[heat] = (ms, it)
        (ms_h, it), (ms_0, _) = res[1], res[0]
        us_it = (ms_h - ms_0) * 1e3 / max(it, 1)
        b = HC_BYTES_PER_CELL_ITER["f64" if prec == PIP_FP64 else "f32"]
        out[name] = {"ms_per_step": ms_h / nsteps, "ms_per_step_without_conduction": ms_0 / nsteps,
                     "cell_updates_per_s": 2048 * 1024 * nsteps / (ms_h * 1e-3),
                     "bicgstab_iterations": it, "iterations_per_step": it / nsteps,
                     "us_per_iteration": us_it,
                     "iteration_gbs": b * 2048 * 1024 / (us_it * 1e-6) / 1e9,
                     "algorithmic_bytes_per_cell_iteration": b}
    # the rounding-only spread: the FP64 path built without FMA contraction against the FMA
    # build, same run; the mixed-vs-FP64 figures above are read against it
    s, Uh, Um = ics.kelvin_helmholtz(2048, 1024, flag_heat=1, kapper=kapper, hc_error=1e-10,
                                     hc_max=5000, fp_exact=1)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.prologue()
        st, t, n, _ = c.run_timed(nsteps=nsteps)
        if st != 0 or n != nsteps:
            raise RuntimeError("C3 FMA-free run ended with status %d after %d steps" % (st, n))
        states["fp64_exact"] = c.download()
    spread = rel_l1_interior(states["fp64_exact"], states["fp64"], 3)
    l1 = rel_l1_interior(states["mixed"], states["fp64"], 3)
    out["l1_fp64_fma_vs_fma_free"] = dict(zip(L1_NAMES[:13], [float(x) for x in spread[:13]]))
    out.update({
        "workload": "2D partially ionised Kelvin-Helmholtz 2048x1024 (+3 ghosts), periodic x, "
                    "reflecting y, IR power law chi=5, kapper=%g (kappa_par ~ T^2.5 along B), "
                    "BiCGstab to relative residual 1e-10, %d steps" % (kapper, nsteps),
        "mixed_over_fp64": out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"],
        "l1_mixed_vs_fp64_max": float(l1[:13].max()),
        "l1_mixed_vs_fp64": dict(zip(L1_NAMES[:13], [float(x) for x in l1[:13]])),
        "how": "device time (CUDA events in the library) of pip_run over %d steps; the solver "
               "time per iteration is (time with conduction - time without) / iterations, and "
               "its GB/s counts the algorithmic bytes of the three BiCGstab kernels" % nsteps})
    return out


# per-variable tables that the printed line carries as their largest entry only (the
# --detail file keeps them whole), and the load-balance terms it leaves to that file
PER_VARIABLE = ("per_variable", "l1_fp64_fma_vs_fma_free", "l1_mixed_vs_fp64")
DETAIL_ONLY = ("busy_us", "ideal_makespan_us", "slots", "longest_run_us", "worst_member",
               "check_s", "cell_updates", "samples", "samples_under_load", "loss",
               "dloss_dcol", "checkpoint_every", "target_backward_over_forward",
               "algorithmic_bytes_per_cell_iteration", "ms_per_step_without_conduction",
               "bicgstab_iterations", "cell_updates_per_s", "step_achieved_gbs",
               "hbm_floor_us_per_step", "checkpointed_forward_ms", "members_checked",
               "max_rel_time_diff", "makespan_us", "after_steps", "bar")


def compact(x, top=True):
    """The printed line: the descriptive strings ("how", "note", the sub-records'
    "workload") dropped -- the module docstring describes each record --, per-variable
    tables cut to their largest entry, and floats rounded to 4 significant digits, so the
    whole line stays short."""
    if isinstance(x, dict):
        out = {}
        for k, v in x.items():
            if k in ("how", "note") or (k == "workload" and not top) or k in DETAIL_ONLY:
                continue
            if not top and k == "gpu_launches" and v == 2 * x.get("steps", -1) + 1:
                continue    # a variant's two launches per step and the final cfl
            if (k in PER_VARIABLE and isinstance(v, dict) and len(v) >= 8 and
                    all(isinstance(t, (int, float)) for t in v.values())):
                name = max(v, key=lambda t: v[t])
                out[k + "_max"] = {"var": name, "value": compact(float(v[name]), False)}
                continue
            out[k] = compact(v, False)
        return out
    if isinstance(x, list):
        return [compact(v, False) for v in x]
    if isinstance(x, float):
        return float("%.4g" % x)
    return x


def rel_l1_interior(a, b, m):
    import numpy as np
    out = []
    for x, y in zip(a, b):
        xi = x[:, m:-m, m:-m].reshape(x.shape[0], -1)
        yi = y[:, m:-m, m:-m].reshape(y.shape[0], -1)
        num = np.abs(xi - yi).sum(axis=1)
        den = np.abs(yi).sum(axis=1)
        out.append(np.where(den > 0, num / np.where(den > 0, den, 1.0), num))
    return np.concatenate(out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=N_GRID, help="grid size (default 1024)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-conduction", action="store_true")
    ap.add_argument("--no-extra-physics", action="store_true")
    ap.add_argument("--decompose", action="store_true",
                    help="run the domain-decomposed step also with one GPU (always with N > 1)")
    ap.add_argument("--detail", default=None,
                    help="also write the full record (descriptions, unrounded) to this file")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.warmup < 3:
        args.warmup = 3

    import torch
    from pip_b200.params import PIP_FP64, PIP_MIXED

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

    def max_over_ranks(x):
        if not dist:
            return x
        tt = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    from pip_b200 import build
    build.build()
    n = args.n
    cells = n * n
    decomposed = world > 1 or args.decompose
    # clocks over the whole measurement (every timed region below lies inside it)
    whole = ClockSampler(local).__enter__()
    if decomposed:
        f64 = measure_decomposed(n, PIP_FP64, args.steps, args.warmup, dist, local, world, rank)
        mix = measure_decomposed(n, PIP_MIXED, args.steps, args.warmup, dist, local, world, rank)
    else:
        f64 = measure(n, PIP_FP64, args.steps, args.warmup, dist, local)
        mix = measure(n, PIP_MIXED, args.steps, args.warmup, dist, local)
    # the FMA-free FP64 flavour: bit for bit the oracle's arithmetic, so it meets the
    # drop-in bar on all 14 fields (the FMA build's psi differs by ~1e-8)
    f64x = None if decomposed else measure(n, PIP_FP64, args.steps, args.warmup, dist, local,
                                           exact=1)
    l1 = rel_l1_interior(mix["state"], f64["state"], 2)
    ms64 = max_over_ranks(f64["ms"])
    msmx = max_over_ranks(mix["ms"])
    v64 = world * cells * args.steps / (ms64 * 1e-3)
    vmx = world * cells * args.steps / (msmx * 1e-3)
    peak, peak_kind = measured_peaks()
    a64 = FP64_BYTES_PER_CELL_STAGE2 * cells / (f64["ms2"] * 1e-3) / 1e9
    amx = MIXED_BYTES_PER_CELL_STAGE2 * cells / (mix["ms2"] * 1e-3) / 1e9
    if decomposed:
        e2e_s, state_bytes = e2e_decomposed(n, PIP_MIXED, args.steps, args.warmup, dist, local,
                                            world, rank)
        how = ("FP32-mixed, decomposed: pip_upload of each rank's block (pinned FP64 host "
               "arrays) + %d device-driven steps (stage, halo, stage, halo, cfl-candidate "
               "allreduce) + pip_download, wall clock, max over ranks" % args.steps)
    else:
        e2e_s, state_bytes = e2e_run(mix["settings"], mix["U"][0], mix["U"][1], args.steps,
                                     args.warmup, dist)
        how = ("FP32-mixed: pip_upload (pinned FP64 host arrays) + pip_run(%d steps) + "
               "pip_download, wall clock around the synchronous C ABI calls" % args.steps)
    e2e_s = max_over_ranks(e2e_s)
    e2e = {"value": world * cells * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": state_bytes / args.steps,
           "d2h_bytes_per_step": state_bytes / args.steps, "how": how}
    if rank != 0:
        whole.__exit__()
        if dist:
            dist.destroy_process_group()
        return 0
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_sample()
        cpu.pop("s_per_step", None)
    adjoint = None if args.no_adjoint else measure_adjoint()
    ensemble = None if args.no_ensemble else measure_ensemble()
    conduction = None if args.no_conduction else measure_conduction()
    alpha_c = resistivity = ionisation = nlevel = None
    if not args.no_extra_physics:
        def variant(what, **kw):
            # a failure here must not cost the headline line
            try:
                return measure_variant(n, 500, ms64 / args.steps, what, **kw)
            except Exception as e:  # noqa: BLE001
                return {"workload": what, "error": str(e)}
        alpha_c = variant("flag_col=5 (set_collisional col_type 4)", flag_col=5)
        resistivity = variant("flag_resi=1, eta_0=1e-4 (resistive_flux)", flag_resi=1,
                              eta_0=1.0e-4)
        ionisation = variant("flag_ir=3 (set_IR type 3 at every stage), T_norm=1.5e4, "
                             "n_norm=1e11, t_IR=10", flag_ir=3, t_norm=1.5e4, n_norm=1.0e11,
                             t_ir=10.0)
        try:
            nlevel = measure_nlevel(n, 200, ms64 / args.steps)
        except Exception as e:  # noqa: BLE001
            nlevel = {"workload": "set_IR type 4", "error": str(e)}
    whole.__exit__()
    line = {
        "metric": METRIC, "value": vmx, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": msmx / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64-mixed", "data": "synthetic",
        "config": {"workload": workload_text(n, world, decomposed),
                   "cells": cells * world,
                   "precision": "FP32-mixed (FP32 fluxes/state, FP64 source and compensated "
                                "RK accumulation)",
                   "l2": "inputs larger than L2 (FP64 state 2 x %.0f MB, mixed 3 x %.0f MB vs "
                         "126 MB L2)" % (state_bytes / 1e6, state_bytes / 2e6),
                   "parallelism": ("y-slab domain decomposition over %d GPU(s)" % world
                                   if decomposed else "single GPU")},
        "fp64": {"value": v64, "ms_per_step": ms64 / args.steps, "dtype": "f64",
                 "roofline": {"bound": "hbm", "achieved": a64, "peak": peak, "unit": "GB/s",
                              "frac": a64 / peak,
                              "traffic": ncu_traffic("stage2_fp64_ot1024"),
                              "algorithmic_bytes_per_cell": FP64_BYTES_PER_CELL_STAGE2,
                              "ms_stage1": f64["ms1"], "ms_stage2": f64["ms2"],
                              "fp64_pipe": {
                                  "floor_us_per_step": FP64_PIPE_US_PER_STEP,
                                  "frac": FP64_PIPE_US_PER_STEP / (f64["ms"] / args.steps * 1e3),
                                  "hbm_floor_us_per_step": FP64_BYTES_PER_CELL_STEP * cells
                                  / (peak * 1e9) * 1e6,
                                  "note": "the FP64 pipe, not HBM, bounds the FP64 stage kernels: "
                                          "its busy time per step (ncu) exceeds the HBM floor "
                                          "~2.6x, so HBM frac cannot pass ~0.38"}},
                 "gpu_launches": f64["launches"], "clocks": f64["clocks"]},
        "fp64_fma_free": None if f64x is None else {
            "value": cells * args.steps / (f64x["ms"] * 1e-3),
            "ms_per_step": f64x["ms"] / args.steps, "ms_stage1": f64x["ms1"],
            "ms_stage2": f64x["ms2"]},
        "mixed_over_fp64": vmx / v64,
        "mixed_over_fp64_fma_free": None if f64x is None else f64x["ms"] / mix["ms"],
        "l1_mixed_vs_fp64": {
            "max_physical": float(max(l1[:5].max(), l1[5:13].max())),
            "psi": float(l1[13]),
            "bar": 1e-5,
            "pass": bool(l1.max() <= 1e-5),
            "pass_physical": bool(max(l1[:5].max(), l1[5:13].max()) <= 1e-5),
            "per_variable": dict(zip(L1_NAMES, [float(x) for x in l1])),
            "after_steps": args.warmup + args.steps,
            "note": "pass is over all 14 stored fields; pass_physical over the 13 physical "
                    "fields (8 MHD + 5 hydro) without the Dedner potential psi, which "
                    "amplifies white noise in B ~1e7-fold (tests/psi_sensitivity.py)"},
        "roofline": {"bound": "hbm", "achieved": amx, "peak": peak, "unit": "GB/s",
                     "frac": amx / peak, "traffic": ncu_traffic("stage2_mixed_ot1024"),
                     "kernel": "mixed stage_kernel<2,9,2> (stage 2: fluxes+source+update+cfl)",
                     "algorithmic_bytes_per_cell": MIXED_BYTES_PER_CELL_STAGE2,
                     "peak_kind": peak_kind, "ms_stage1": mix["ms1"], "ms_stage2": mix["ms2"],
                     "step_achieved_gbs": MIXED_BYTES_PER_CELL_STEP * cells / (mix["msstep"] * 1e-3) / 1e9},
        "cpu_baseline": cpu,
        "adjoint": adjoint,
        "ensemble": ensemble,
        "conduction": conduction,
        "alpha_c_per_cell": alpha_c,
        "resistivity": resistivity,
        "ionisation_recombination": ionisation,
        "nlevel_hydrogen": nlevel,
        "e2e": e2e,
        "gpu_launches": mix["launches"],
        "clocks": whole.summary(),
    }
    if args.detail:
        with open(args.detail, "w") as f:
            json.dump(line, f, indent=1)
    print(json.dumps(compact(line)), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
