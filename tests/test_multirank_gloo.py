"""Replica aggregation of bench.py across ranks, on CPU with the gloo backend (world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms, units, launches = bench.reduce_over_ranks(dist, "cpu", 10.0 + rank, 1000.0 * (rank + 1),
                                                  7 + rank)
    out[rank] = (ms, units, launches)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_max_time_sum_units():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        ms, units, launches = out[r]
        assert ms == 11.0          # max over ranks
        assert units == 3000.0     # sum over ranks
        assert launches == 15
