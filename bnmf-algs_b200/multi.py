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


def row_shards(x, world):
    """[i0, i1) of every rank for a row-sharded solve: contiguous blocks whose
    sizes differ by at most one row."""
    if world < 1 or x < world:
        raise ValueError("need at least one row per shard")
    base, extra = divmod(x, world)
    out, i0 = [], 0
    for r in range(world):
        i1 = i0 + base + (1 if r < extra else 0)
        out.append((i0, i1))
        i0 = i1
    return out


class Shard:
    """One row block of a sharded instance: its plan (or any object with the
    plan's shard_* methods) and its device buffers.  red holds
    plan.shard_red_size() FP64 values."""

    def __init__(self, plan, dX, dalpha, dbeta, dS, red):
        self.plan, self.dX, self.dalpha, self.dbeta, self.dS, self.red = (
            plan, dX, dalpha, dbeta, dS, red)


def sharded_solve(shards, iters, psi_mode, eps, allreduce):
    """bld_mult over row shards.  Only the sums over rows cross shards (S_+jk
    and sum_i alpha_eph, y*z + z values per iteration): every shard sweeps
    its rows into its red, allreduce(reds) sums the reds of all shards of the
    job in place (one all-reduce per iteration across ranks; a sum over the
    list for several shards in one process), and every shard tabulates the
    shared digamma values from the global sums.  Every rank takes the same
    collective steps in the same order."""
    reds = [sh.red for sh in shards]
    for sh in shards:
        sh.plan.shard_sums(sh.dS, sh.dalpha, sh.red, psi_mode)
    allreduce(reds)
    for sh in shards:
        sh.plan.shard_finish(sh.dbeta, sh.red, psi_mode)
    for it in range(iters):
        for sh in shards:
            sh.plan.shard_update(sh.dX, sh.dS, sh.dalpha, sh.red, psi_mode, eps)
        allreduce(reds)
        if it + 1 < iters:
            for sh in shards:
                sh.plan.shard_finish(sh.dbeta, sh.red, psi_mode)


def collective_allreduce(dist):
    """allreduce for sharded_solve with one shard per rank (NCCL or gloo)."""
    def reduce(reds):
        for r in reds:
            dist.all_reduce(r, op=dist.ReduceOp.SUM)
    return reduce


def local_allreduce(reds):
    """allreduce for several shards in one process: the sum in shard order,
    written back to every shard's buffer."""
    total = reds[0].clone()
    for r in reds[1:]:
        total += r
    for r in reds:
        r.copy_(total)
