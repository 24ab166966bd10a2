"""World-size-2 gloo tests (CPU) of the multi-GPU host logic: the batch
partition is disjoint, complete and identical on every rank without
communication, and throughput aggregates as total work over the slowest rank."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_package


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        load_package()
        import bnmf_algs_b200.multi as M
        import bnmf_algs_b200.workloads as W
        shapes = W.batch_shapes(512, 3)
        mine = M.shard_instances(shapes, world, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        work = sum(shapes[i][0] * shapes[i][1] * shapes[i][2] for i in mine)
        seconds = 1.0 + rank  # rank 1 is the slowest
        thr = M.aggregate_throughput(work, seconds, dist)
        q.put((rank, gathered, work, thr))
    finally:
        dist.destroy_process_group()


def test_batch_partition_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    g0, g1 = res[0][1], res[1][1]
    assert g0 == g1                      # every rank computed the same partition
    all_idx = sorted(g0[0] + g0[1])
    assert all_idx == list(range(512))   # complete and disjoint
    w0, w1 = res[0][2], res[1][2]
    assert abs(w0 - w1) / max(w0, w1) < 0.05   # LPT balances the work
    total = w0 + w1
    for r in res:
        assert abs(r[3] - total / 2.0) < 1e-6 * total   # slowest rank took 2 s


def test_partition_single_process():
    load_package()
    import bnmf_algs_b200.multi as M
    shapes = [(10, 10, 4), (20, 20, 4), (5, 5, 4)]
    assert M.shard_instances(shapes, 1, 0) == [0, 1, 2]
    with pytest.raises(ValueError):
        M.shard_instances(shapes, 2, 2)
    assert M.aggregate_throughput(10.0, 2.0) == 5.0
