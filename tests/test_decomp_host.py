"""Domain decomposition (pip_b200.decomp, the MPI layer of MPI_rot.f90) on the CPU: the
split, neighbour tables and coordinates of set_mpi / set_mpi_neighbor / set_coordinate,
scatter/gather, and whole decomposed runs -- blocks on the oracle, exchanging halos through
a world-size-2 gloo process group or inside one process -- against the single-domain
oracle run, bitwise (the split is into powers of two, so every block's grid spacing is the
single grid's)."""
import multiprocessing as mp
import socket

import numpy as np
import pytest

import decomp_worker
from decomp_cases import make_case
from oracle import oracle as O
from oracle_block import OracleBlock
from pip_b200 import decomp, ics, output


def single_domain(case, nsteps):
    s, Uh, Um = make_case(case)
    o = O.Oracle(s, Uh, Um)
    st, t, n, hist = o.run(nsteps=nsteps, max_hist=nsteps)
    uh, um = o.state()
    o.close()
    assert st == 0 and n == nsteps
    return s, uh, um, hist


def test_block_neighbours_and_coordinates():
    s, _, _ = ics.orszag_tang(16)            # periodic: the ends wrap around
    assert [decomp.block_of(s, 4, r).neighbor for r in range(4)] == [
        (-1, -1, 3, 1), (-1, -1, 0, 2), (-1, -1, 1, 3), (-1, -1, 2, 0)]
    s2, _, _ = ics.kelvin_helmholtz(16, 16)  # reflecting in y: physical ends
    assert [decomp.block_of(s2, 2, r).neighbor for r in range(2)] == [(-1, -1, -1, 1), (-1, -1, 0, -1)]
    s1, _, _ = ics.brio_wu(64)               # 1D splits along x
    assert decomp.block_of(s1, 2, 1).neighbor == (0, -1, -1, -1)
    assert decomp.block_of(s, 1, 0).neighbor == (-1, -1, -1, -1)
    # the blocks' grid spacing and cell centres are the single grid's (powers of two)
    _, y, _, _, dy, _ = s.coordinates()
    m = s.margin[1]
    for r in range(4):
        b = decomp.block_of(s, 4, r)
        _, yb, _, _, dyb, _ = b.settings.coordinates()
        assert np.array_equal(dyb, dy[: dyb.size])
        assert np.allclose(yb, y[b.lo: b.lo + b.n + 2 * m], rtol=0, atol=1e-15)
    with pytest.raises(ValueError):
        decomp.block_of(s, 3, 0)


@pytest.mark.parametrize("case,world", [("ot", 2), ("ot", 4), ("bw", 4)])
def test_scatter_gather_round_trip(case, world):
    s, Uh, Um = make_case(case)
    parts = [decomp.scatter(s, Um, world, r) for r in range(world)]
    assert np.array_equal(decomp.gather(s, parts), Um)


def local_run(case, world, nsteps):
    s, Uh, Um = make_case(case)
    engines = [OracleBlock(decomp.block_of(s, world, r), decomp.scatter(s, Uh, world, r),
                           decomp.scatter(s, Um, world, r)) for r in range(world)]
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    st = run.run(nsteps)
    states = [e.download() for e in engines]
    run.close()
    uh = decomp.gather(s, [a for a, _ in states])
    um = decomp.gather(s, [b for _, b in states])
    return st, run.dt_history, uh, um


@pytest.mark.parametrize("case,world", [("ot", 2), ("ot", 4), ("ot_generic", 2), ("kh", 2),
                                        ("kh", 4), ("bw", 2), ("bw", 4), ("ot_col", 4),
                                        ("kh_col", 2), ("ot_resi", 4)])
def test_blocks_in_one_process_match_single_domain(case, world):
    nsteps = 6
    s, uh, um, hist = single_domain(case, nsteps)
    st, dts, gh, gm = local_run(case, world, nsteps)
    assert st == 0
    assert np.array_equal(np.array(dts), hist)
    assert np.array_equal(gh, uh) and np.array_equal(gm, um)


def _free_port():
    with socket.socket() as k:
        k.bind(("127.0.0.1", 0))
        return k.getsockname()[1]


@pytest.mark.parametrize("case", ["ot", "kh", "bw", "ot_resi", "kh_ir1", "kh_ir3"])
def test_two_gloo_ranks_match_single_domain(case):
    nsteps = 5
    s, uh, um, hist = single_domain(case, nsteps)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=decomp_worker.rank_main, args=(r, 2, port, case, nsteps, q))
             for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for rank, st, dts, _, _ in got:
        assert st == 0, (rank, st, dts)
        assert np.array_equal(np.array(dts), hist)
    gh = decomp.gather(s, [g[3] for g in got])
    gm = decomp.gather(s, [g[4] for g in got])
    assert np.array_equal(gh, uh) and np.array_equal(gm, um)


@pytest.mark.parametrize("case", ["kh", "ot_col"])
def test_decomposed_output_is_the_single_domain_output(tmp_path, case):
    """Each block writes its hyperslab of output 1 after 4 steps; the file is the one the
    single-domain run writes (with alpha_c per cell, its field too)."""
    s, Uh, Um = make_case(case)
    o = O.Oracle(s, Uh, Um)
    o.run(nsteps=4)
    oh, om = o.state()
    ac = o.alpha_c() if s.flag_col >= 2 else None
    ref = output.write_output(str(tmp_path / "one"), 1, s, o.time, oh, om, ac)
    o.close()
    engines = [OracleBlock(decomp.block_of(s, 4, r), decomp.scatter(s, Uh, 4, r),
                           decomp.scatter(s, Um, 4, r)) for r in range(4)]
    run = decomp.DecomposedRun(engines, decomp.LocalComm(), divb=s.divb == 1)
    assert run.run(4) == 0
    run.write_output(str(tmp_path / "blocks"), 1, s)
    run.close()
    assert open(ref, "rb").read() == open(str(tmp_path / "blocks" / "t0001.bin"), "rb").read()


def test_candidate_reduction_over_two_gloo_ranks():
    """The device-driven loop's reduction (TorchComm.reduce_candidates): MIN of the dt words
    and MAX of the rho/IR-rate words as int64 bit patterns equal the doubles' MIN/MAX."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=decomp_worker.reduce_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted((q.get(timeout=120) for _ in procs), key=lambda x: x[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(not isinstance(g[1], str) for g in got), got
    want_min = np.minimum(got[0][1], got[1][1])
    want_max = np.maximum(got[0][2], got[1][2])
    for g in got:
        assert np.array_equal(g[3], want_min) and np.array_equal(g[4], want_max)


@pytest.mark.parametrize("case,world", [("kh_hc", 2), ("kh_hc", 4), ("kh_hc_generic", 1),
                                        ("kh_hc_generic", 2), ("kh_hc_generic", 4)])
def test_conduction_blocks_match_single_domain(case, world):
    """post_step's implicit conduction of a decomposed run (BiCGstabMPI in phases, global
    scalars, one row of r and Ap exchanged per face) against the single domain: one block
    (no neighbours) conducts inside its stage as the single domain does, bitwise; more blocks
    group the dot products by rank, so the iterates agree to rounding (and the iteration
    count near the 1e-12 stop may differ)."""
    nsteps = 4
    s, uh, um, hist = single_domain(case, nsteps)
    st, dts, gh, gm = local_run(case, world, nsteps)
    assert st == 0
    if world == 1:
        assert np.array_equal(np.array(dts), hist)
        assert np.array_equal(gh, uh) and np.array_equal(gm, um)
        return
    assert np.allclose(np.array(dts), hist, rtol=1e-11, atol=0)
    rel = max(np.abs(gh - uh).max() / np.abs(uh).max(), np.abs(gm - um).max() / np.abs(um).max())
    assert rel <= 1e-11, rel


def test_conduction_over_two_gloo_ranks():
    """The same through a world-size-2 gloo group: the scalars by all_reduce(SUM), the rows
    by point-to-point messages."""
    case, nsteps = "kh_hc_generic", 3
    s, uh, um, hist = single_domain(case, nsteps)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=decomp_worker.rank_main, args=(r, 2, port, case, nsteps, q))
             for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for rank, st, dts, _, _ in got:
        assert st == 0, (rank, st, dts)
        assert np.allclose(np.array(dts), hist, rtol=1e-11, atol=0)
    gh = decomp.gather(s, [g[3] for g in got])
    gm = decomp.gather(s, [g[4] for g in got])
    rel = max(np.abs(gh - uh).max() / np.abs(uh).max(), np.abs(gm - um).max() / np.abs(um).max())
    assert rel <= 1e-11, rel
