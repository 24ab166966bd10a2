"""Multi-GPU host logic: one process per GPU, no data-path collective.

The plain solve runs as independent replicas (one per rank).  A batch of
independent instances is partitioned across ranks by work (x*y*z) with a
deterministic longest-processing-time assignment, so every rank computes the
same partition without communicating.  Throughput is the work of all ranks
divided by the slowest rank's time (max over ranks).
"""

import heapq


def shard_instances(shapes, world, rank):
    """Indices of the instances rank `rank` of `world` solves (LPT by x*y*z)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    order = sorted(range(len(shapes)), key=lambda i: (-shapes[i][0] * shapes[i][1] * shapes[i][2], i))
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(shapes)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        x, y, z = shapes[i]
        heapq.heappush(heap, (load + x * y * z, r))
    return [i for i in range(len(shapes)) if owner[i] == rank]


def max_over_ranks(value, dist=None, device=None):
    """max of a per-rank float over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device=None):
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate_throughput(units, seconds, dist=None, device=None):
    """(total units over ranks) / (slowest rank's seconds)."""
    total = sum_over_ranks(units, dist, device)
    slowest = max_over_ranks(seconds, dist, device)
    return total / slowest
