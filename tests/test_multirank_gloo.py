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


def _shard_worker(rank, world, port, q):
    import torch.distributed as dist
    from emerge_engine_b200.sharding import shard_scenes
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    costs = [((k * 7919) % 97 + 1) * 1000 for k in range(40)]
    mine = shard_scenes(costs, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    q.put((rank, got))
    dist.destroy_process_group()


def test_scene_sharding_is_consistent_and_balanced():
    """Every rank derives the same placement; each scene lands on exactly one rank and the
    most loaded rank is within 4/3 of the average plus one scene."""
    import multiprocessing as mp
    import socket
    from emerge_engine_b200.sharding import shard_loads, shard_scenes
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 3
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    views = [r[1] for r in results]
    assert all(v == views[0] for v in views)
    flat = sorted(i for shard in views[0] for i in shard)
    assert flat == list(range(40))
    costs = [((k * 7919) % 97 + 1) * 1000 for k in range(40)]
    loads = shard_loads(costs, shard_scenes(costs, world))
    assert max(loads) <= 4.0 / 3.0 * sum(costs) / world + max(costs)
