"""Multi-rank path of bench.py on the CPU (gloo, world size 2): replicas are
independent, the whole-job totals sum the detected symbols over the ranks and
take the slowest rank's time (the N > 1 contract: value = all ranks' symbols
/ max time)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

from tests.conftest import ROOT


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    import bench
    from libapsm_b200 import synth

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        dets = synth.config2_detectors(3, seed=2 + rank, data=(1000, 1200), pilots=(200, 220))
        sym = sum(d.S for d in dets)
        res = bench.replica_totals(sym, 10.0 + rank, 20.0 - rank, world, "cpu")
        out[rank] = (sym, res)
    finally:
        dist.destroy_process_group()


def test_replica_totals_two_ranks():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        got = dict(out)
    sym0, (tot0, t0, e0) = got[0]
    sym1, (tot1, t1, e1) = got[1]
    assert sym0 != sym1  # each replica draws its own detectors
    assert tot0 == tot1 == sym0 + sym1
    assert (t0, e0) == (t1, e1) == (11.0, 20.0)
