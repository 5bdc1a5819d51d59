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
