"""Child process of the world-size-2 decomposition tests: one rank of a gloo process group
stepping its block on the oracle through pip_b200.decomp, results back over a queue."""
import os
import sys


def rank_main(rank, world, port, case, nsteps, q):
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (here, os.path.dirname(here)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    from pip_b200 import decomp
    from oracle_block import OracleBlock
    from decomp_cases import make_case
    try:
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                                world_size=world, timeout=datetime.timedelta(seconds=60))
        s, Uh, Um = make_case(case)
        b = decomp.block_of(s, world, rank)
        eng = OracleBlock(b, decomp.scatter(s, Uh, world, rank), decomp.scatter(s, Um, world, rank))
        run = decomp.DecomposedRun([eng], decomp.TorchComm("cpu"), divb=s.divb == 1)
        st = run.run(nsteps)
        uh, um = eng.download()
        q.put((rank, st, run.dt_history, uh, um))
        eng.close()
        dist.destroy_process_group()
    except Exception as e:   # reported to the parent, which fails the test
        q.put((rank, "error", repr(e), None, None))


def reduce_main(rank, world, port, q):
    """cfl-candidate reduction of the device-driven loop over a gloo group: each rank holds
    its candidates as int64 bit patterns of positive doubles (dt words to MIN, rho/IR-rate
    words to MAX); the reduced words must be the bit patterns of the doubles' MIN/MAX."""
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (here, os.path.dirname(here)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    from pip_b200 import decomp
    try:
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                                world_size=world, timeout=datetime.timedelta(seconds=60))
        comm = decomp.TorchComm("cpu")
        rng = np.random.default_rng(100 + rank)
        dt = rng.uniform(1e-5, 1e-2, 2)
        mx = rng.uniform(0.0, 1e4, 4)
        t_min = torch.from_numpy(dt.view(np.int64).copy())
        t_max = torch.from_numpy(mx.view(np.int64).copy())
        comm.reduce_candidates([(t_min, t_max)])
        comm.barrier()
        q.put((rank, dt, mx, t_min.numpy().view(np.float64).copy(),
               t_max.numpy().view(np.float64).copy()))
        dist.destroy_process_group()
    except Exception as e:
        q.put((rank, "error", repr(e), None, None))


def device_rank_main(rank, world, port, case, nsteps, device_loop, q):
    """One rank of a gloo group stepping its block on a GPU context (cuda:0, shared by the
    ranks: the host sequences each rank's launches and the messages go through host
    copies, so no kernel waits for another rank)."""
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (here, os.path.dirname(here)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime
    import torch
    import torch.distributed as dist
    from pip_b200 import decomp
    from decomp_cases import make_case
    try:
        torch.cuda.set_device(0)
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                                world_size=world, timeout=datetime.timedelta(seconds=60))
        s, Uh, Um = make_case(case)
        b = decomp.block_of(s, world, rank)
        eng = decomp.DeviceBlock(b, decomp.scatter(s, Uh, world, rank),
                                 decomp.scatter(s, Um, world, rank))
        run = decomp.DecomposedRun([eng], decomp.TorchComm("cpu", staged=True),
                                   divb=s.divb == 1)
        st = run.run_device(nsteps) if device_loop else run.run(nsteps)
        uh, um = eng.download()
        q.put((rank, st, run.dt_history, uh, um))
        run.close()
        dist.destroy_process_group()
    except Exception as e:   # reported to the parent, which fails the test
        q.put((rank, "error", repr(e), None, None))

