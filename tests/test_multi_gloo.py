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


class _CpuShard:
    """The shard steps of a plan, restated on the CPU with the oracle's digamma
    (test stand-in for the GPU plan, so that the collective schedule of
    multi.sharded_solve runs over real gloo ranks)."""

    def __init__(self, oracle, y, z):
        self.o, self.y, self.z = oracle, y, z

    def _sums(self, S, alpha, red):
        pjk = S.sum(0)
        self.alpha_eph = S.sum(1) + alpha[:, None]
        r = red.numpy()
        r[: self.y * self.z] = pjk.ravel()
        r[self.y * self.z:] = self.alpha_eph.sum(0)

    def shard_sums(self, S, alpha, red, psi_mode):
        self._sums(S, alpha, red)

    def shard_finish(self, beta, red, psi_mode):
        r = red.numpy()
        yz = self.y * self.z
        self.psiB = self.o.psi_array(r[:yz].reshape(self.y, self.z) + beta[None, :])
        self.psiAS = self.o.psi_array(r[yz:])
        self.psiA = self.o.psi_array(self.alpha_eph)

    def shard_update(self, X, S, alpha, red, psi_mode, eps):
        gp = self.psiB[None, :, :] - self.o.psi_array(S + 1.0)
        gm = self.psiAS[None, :] - self.psiA
        xr = 1.0 / (X + eps)
        nom = (S * gm[:, None, :]).sum(2) * xr
        den = (S * gp).sum(2) * xr
        ijp = S.sum(2)
        S[...] = S * (gp + nom[..., None]) * (X / (ijp + eps))[..., None] / (
            gm[:, None, :] + den[..., None] + eps)
        self._sums(S, alpha, red)


def _shard_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        load_package()
        import sys
        import numpy as np
        sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
        import oracle as O
        import bnmf_algs_b200.multi as M
        import bnmf_algs_b200.workloads as W
        prob = W.plain_small(3)
        X, z = prob["X"], prob["z"]
        x, y = X.shape
        S0 = O.init_S(X, z, 2)
        i0, i1 = M.row_shards(x, world)[rank]
        red = torch.empty(y * z + z, dtype=torch.float64)
        sh = M.Shard(_CpuShard(O, y, z), X[i0:i1].copy(), prob["alpha"][i0:i1].copy(),
                     prob["beta"].copy(), S0[i0:i1].copy(), red)
        M.sharded_solve([sh], 10, O.PSI_APPR, 1e-50, M.collective_allreduce(dist))
        parts = [None] * world
        dist.all_gather_object(parts, sh.dS)
        q.put((rank, np.concatenate(parts, axis=0), X, z, prob, S0))
    finally:
        dist.destroy_process_group()


def test_row_sharded_solve_over_two_gloo_ranks():
    """multi.sharded_solve with one row shard per gloo rank and one all-reduce
    per iteration gives the unsharded oracle solve (to summation order)."""
    import sys
    import numpy as np
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    S, X, z, prob, S0 = res[0][1], res[0][2], res[0][3], res[0][4], res[0][5]
    np.testing.assert_array_equal(S, res[1][1])  # both ranks hold the same gathered S
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    import oracle as O
    ref = O.bld_mult(X, z, prob["alpha"], prob["beta"], 10, O.PSI_APPR, 1e-50, S0=S0)
    assert np.abs(S - ref).max() <= 1e-10 * np.abs(ref).max()


def test_row_shards_cover_rows():
    load_package()
    import bnmf_algs_b200.multi as M
    assert M.row_shards(10, 3) == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError):
        M.row_shards(2, 3)
