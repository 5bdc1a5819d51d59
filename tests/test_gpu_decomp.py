"""Domain decomposition on the device: blocks on GPU contexts (pip_set_neighbors,
pip_stage, pip_halo_pack / pip_halo_unpack) stepped by pip_b200.decomp.  The run here has
every block in one process on one GPU (the host sequences the blocks' launches; nothing
on the device waits for another block), exchanging halos by device copies; the same
driver over torch.distributed/NCCL moves the same buffers between GPUs.  Checked against
the single-block run of the same driver (bitwise: the per-cell arithmetic does not depend
on the split), against pip_run, and against the single-domain oracle."""
import ctypes

import numpy as np
import pytest
import torch

from decomp_cases import make_case
from helpers import interior, rel_l1
from oracle import oracle as O
from pip_b200 import capi, decomp, ics
from pip_b200.params import PIP_FP64, PIP_MIXED

pytestmark = pytest.mark.gpu


def device_run(s, Uh, Um, world, nsteps):
    engines = [decomp.DeviceBlock(decomp.block_of(s, world, r), decomp.scatter(s, Uh, world, r),
                                  decomp.scatter(s, Um, world, r)) for r in range(world)]
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    st = run.run(nsteps)
    states = [e.download() for e in engines]
    run.close()
    return (st, run.dt_history, decomp.gather(s, [a for a, _ in states]),
            decomp.gather(s, [b for _, b in states]))


def test_halo_pack_unpack_layout(gpu_lib):
    s, Uh, Um = make_case("ot_generic")
    b = decomp.block_of(s, 2, 0)
    uh, um = decomp.scatter(s, Uh, 2, 0), decomp.scatter(s, Um, 2, 0)
    U = np.concatenate([um, uh], axis=0)
    ix, jx, _ = b.settings.shape
    m = b.settings.margin[1]
    with capi.Context(b.settings) as c:
        c.set_neighbors(b.neighbor)
        c.upload(uh, um)
        assert c.halo_bytes(2) == 8 * U.shape[0] * m * ix
        buf = torch.empty(c.halo_bytes(2), dtype=torch.uint8, device="cuda")
        for face, rows in ((2, slice(m, 2 * m)), (3, slice(jx - 2 * m, jx - m))):
            n = c.halo_pack(face, buf.data_ptr())
            torch.cuda.synchronize()                 # the pack is queued on the context stream
            got = buf[:n].cpu().numpy().view(np.float64).reshape(U.shape[0], m, ix)
            assert np.array_equal(got, U[:, rows, :])
        bufx = torch.empty(c.halo_bytes(0), dtype=torch.uint8, device="cuda")
        n = c.halo_pack(1, bufx.data_ptr())
        torch.cuda.synchronize()
        got = bufx[:n].cpu().numpy().view(np.float64).reshape(U.shape[0], m, jx)
        assert np.array_equal(got, U[:, :, ix - 2 * m: ix - m].transpose(0, 2, 1))
        # a message into the lower ghost rows, nothing else touched
        msg = np.arange(U.shape[0] * m * ix, dtype=np.float64)
        t = torch.from_numpy(msg).cuda().view(torch.uint8)
        torch.cuda.synchronize()                     # the message is in place before unpacking
        c.halo_unpack(2, t.data_ptr(), t.numel())
        gh, gm = c.download()
        G = np.concatenate([gm, gh], axis=0)
        assert np.array_equal(G[:, :m, :], msg.reshape(U.shape[0], m, ix))
        assert np.array_equal(G[:, m:, :], U[:, m:, :])


@pytest.mark.parametrize("case,world", [("ot", 2), ("ot", 4), ("ot_generic", 2), ("kh", 4),
                                        ("bw", 4)])
def test_blocks_match_single_block(gpu_lib, case, world):
    nsteps = 8
    s, Uh, Um = make_case(case)
    st1, dt1, h1, m1 = device_run(s, Uh, Um, 1, nsteps)
    stn, dtn, hn, mn = device_run(s, Uh, Um, world, nsteps)
    assert st1 == 0 and stn == 0
    assert dtn == dt1
    assert np.array_equal(hn, h1) and np.array_equal(mn, m1)
    # the single block through pip_stage is the step of pip_run
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st, t, n = c.run(nsteps=nsteps)
        rh, rm = c.download()
    assert st == 0 and n == nsteps
    assert abs(t - sum(dt1)) <= 1e-14 * t
    assert max(rel_l1(interior(h1, s), interior(rh, s)).max(),
               rel_l1(interior(m1, s), interior(rm, s)).max()) <= 1e-12
    # and the oracle's single-domain run
    o = O.Oracle(s, Uh, Um)
    st_o, t_o, n_o, hist = o.run(nsteps=nsteps, max_hist=nsteps)
    oh, om = o.state()
    o.close()
    np.testing.assert_allclose(np.array(dtn), hist, rtol=1e-10, atol=0)
    assert max(rel_l1(interior(hn, s), interior(oh, s)).max(),
               rel_l1(interior(mn, s), interior(om, s)).max()) <= 1e-10


def test_mixed_blocks_match_single_block(gpu_lib):
    s, Uh, Um = ics.orszag_tang(32, precision=PIP_MIXED)
    st1, dt1, h1, m1 = device_run(s, Uh, Um, 1, 6)
    st2, dt2, h2, m2 = device_run(s, Uh, Um, 4, 6)
    assert st1 == 0 and st2 == 0 and dt1 == dt2
    assert np.array_equal(h2, h1) and np.array_equal(m2, m1)


def test_decomposition_rejects(gpu_lib):
    s, Uh, Um = ics.orszag_tang(16)
    b = decomp.block_of(s, 2, 0)
    with capi.Context(b.settings) as c:
        c.set_neighbors(b.neighbor)
        c.upload(decomp.scatter(s, Uh, 2, 0), decomp.scatter(s, Um, 2, 0))
        with pytest.raises(capi.PipError) as e:
            c.run_solver(1e-4)                       # pip_step cannot exchange mid-step
        assert e.value.code == capi.PIP_ERR_STATE
        with pytest.raises(capi.PipError) as e:
            c.run(nsteps=1)
        assert e.value.code == capi.PIP_ERR_STATE
        with pytest.raises(capi.PipError) as e:
            c.stage(2, 1e-4, 0.0)                    # stage 2 before stage 1
        assert e.value.code == capi.PIP_ERR_STATE
        with pytest.raises(capi.PipError) as e:
            c.set_neighbors([0, -1, -1, -1])         # x is not split, but accepted ...
            c.set_neighbors([-2, -1, -1, -1])        # ... a rank below -1 is not
        assert e.value.code == capi.PIP_ERR_PARAM
    s3, _, _ = ics.kelvin_helmholtz(16, 16, flag_heat=1, kapper=0.1)
    with capi.Context(s3) as c:
        with pytest.raises(capi.PipError) as e:
            c.set_neighbors([1, -1, -1, -1])         # conduction splits along y only
        assert e.value.code == capi.PIP_ERR_PARAM
        c.set_neighbors([-1, -1, 1, 1])


def device_loop_run(s, Uh, Um, world, nsteps, overlap=False):
    engines = [decomp.DeviceBlock(decomp.block_of(s, world, r), decomp.scatter(s, Uh, world, r),
                                  decomp.scatter(s, Um, world, r)) for r in range(world)]
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    st = run.run_device(nsteps, check_every=4, overlap=overlap)
    states = [e.download() for e in engines]
    run.close()
    return (st, run.time, run.steps, decomp.gather(s, [a for a, _ in states]),
            decomp.gather(s, [b for _, b in states]))


@pytest.mark.parametrize("case,world", [("ot", 2), ("ot", 4), ("ot_generic", 4), ("kh", 4),
                                        ("bw", 4)])
def test_device_loop_blocks_match_pip_run(gpu_lib, case, world):
    """pip_dev_*: dt, cmax and time stay on the device, the candidates are reduced over the
    blocks between steps; the result is pip_run's on the whole grid, bitwise."""
    nsteps = 10
    s, Uh, Um = make_case(case)
    st, t, n, hn, mn = device_loop_run(s, Uh, Um, world, nsteps)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st1, t1, n1 = c.run(nsteps=nsteps)
        rh, rm = c.download()
    assert st == 0 and st1 == 0 and n == n1 == nsteps
    assert t == t1
    assert np.array_equal(hn, rh) and np.array_equal(mn, rm)


def test_device_loop_mixed_matches_pip_run(gpu_lib):
    s, Uh, Um = ics.orszag_tang(32, precision=PIP_MIXED)
    st, t, n, hn, mn = device_loop_run(s, Uh, Um, 4, 9)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st1, t1, n1 = c.run(nsteps=9)
        rh, rm = c.download()
    assert st == 0 and n == 9 and t == t1
    assert np.array_equal(hn, rh) and np.array_equal(mn, rm)


@pytest.mark.parametrize("precision", [PIP_FP64, PIP_MIXED])
@pytest.mark.parametrize("world", [2, 4])
def test_device_loop_overlapped_exchange_matches_pip_run(gpu_lib, precision, world):
    """The y exchange overlapped with each stage: the first and last tile rows first, the
    exchange on its own stream while the middle rows compute.  Blocks of 64 or 32 rows hold
    several tile rows (the mixed kernels' 14-row tiles: 2 with no middle row at 32), so both
    launches of a stage do work; bitwise pip_run's result (power-of-two splits keep the
    blocks' grid spacing equal to the single grid's)."""
    s, Uh, Um = ics.orszag_tang(128, precision=precision)
    st, t, n, hn, mn = device_loop_run(s, Uh, Um, world, 12, overlap=True)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st1, t1, n1 = c.run(nsteps=12)
        rh, rm = c.download()
    assert st == 0 and st1 == 0 and n == n1 == 12 and t == t1
    assert np.array_equal(hn, rh) and np.array_equal(mn, rm)


def test_split_stage_enforces_its_order(gpu_lib):
    s, Uh, Um = ics.orszag_tang(32)
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        c.dev_begin(nsteps=2)
        L = capi.lib()
        bs = ctypes.c_void_p()
        assert L.pip_dev_stage_split(c.h, 2, ctypes.byref(bs)) == capi.PIP_ERR_STATE
        assert L.pip_dev_stage_split(c.h, 1, ctypes.byref(bs)) == capi.PIP_OK and bs.value
        assert L.pip_dev_stage_split(c.h, 2, ctypes.byref(bs)) == capi.PIP_OK
        c.dev_poll()


@pytest.mark.parametrize("case,world", [("kh_hc", 2), ("kh_hc_generic", 1), ("kh_hc_generic", 2),
                                        ("kh_hc_generic", 4)])
def test_conduction_blocks_match_single_domain(gpu_lib, case, world):
    """post_step's conduction of a decomposed run on device blocks (pip_hcd_*: BiCGstabMPI's
    phases with global scalars, rows of r and Ap exchanged) against pip_run of the whole grid
    and against the single-domain oracle.  The dot products group by block, so the iterates
    agree to rounding; one block (no neighbours) conducts inside its stage, as pip_run."""
    nsteps = 4
    s, Uh, Um = make_case(case)
    st, dts, gh, gm = device_run(s, Uh, Um, world, nsteps)
    assert st == 0
    with capi.Context(s) as c:
        c.upload(Uh, Um)
        st1, t1, n1 = c.run(nsteps)
        h1, m1 = c.download()
    assert abs(sum(dts) - t1) <= 1e-11 * t1
    e = max(rel_l1(interior(gh, s), interior(h1, s)).max(), rel_l1(interior(gm, s), interior(m1, s)).max())
    assert e <= 1e-11, e
    o = O.Oracle(s, Uh, Um)
    ost, ot, on, _ = o.run(nsteps=nsteps)
    oh, om = o.state()
    o.close()
    e2 = max(rel_l1(interior(gh, s), interior(oh, s)).max(), rel_l1(interior(gm, s), interior(om, s)).max())
    assert e2 <= 1e-10, e2


def _free_port():
    import socket
    with socket.socket() as k:
        k.bind(("127.0.0.1", 0))
        return k.getsockname()[1]


@pytest.mark.parametrize("case,device_loop", [("ot", False), ("kh", True)])
def test_two_processes_over_gloo(gpu_lib, case, device_loop):
    """The transport path of a multi-GPU run with device blocks: two processes in a gloo
    group, each stepping its block on a GPU context (both on this GPU; the host sequences
    each process's launches), halos and cfl reductions through torch.distributed with host
    staging.  Bitwise the single block's result (host-driven) or pip_run's (device loop)."""
    import multiprocessing as mp
    import decomp_worker
    nsteps = 6
    s, Uh, Um = make_case(case)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=decomp_worker.device_rank_main,
                         args=(r, 2, port, case, nsteps, device_loop, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted((q.get(timeout=240) for _ in procs), key=lambda x: x[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for rank, st, dts, _, _ in got:
        assert st == 0, (rank, st, dts)
    hn = decomp.gather(s, [g[3] for g in got])
    mn = decomp.gather(s, [g[4] for g in got])
    if device_loop:
        with capi.Context(s) as c:
            c.upload(Uh, Um)
            st1, t1, n1 = c.run(nsteps=nsteps)
            rh, rm = c.download()
        assert st1 == 0 and n1 == nsteps
    else:
        st1, dt1, rh, rm = device_run(s, Uh, Um, 1, nsteps)
        assert st1 == 0 and got[0][2] == dt1 == got[1][2]
    assert np.array_equal(hn, rh) and np.array_equal(mn, rm)

