"""Target sharding on the CPU: the cut (restated in tests/shard_ref.py) on the
oracle's geometry, and the assembly of sharded outputs over a 2-rank gloo
group (pacman_b200.distributed.assemble)."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from pacman_b200 import distributed as pdist
from pacman_b200 import workloads as W
from tests import shard_ref


def _case():
    rng = np.random.default_rng(4)
    S = np.concatenate([rng.random((3000, 3)), 0.5 + 0.03 * rng.standard_normal((1500, 3))])
    T = rng.random((3500, 3))
    return S, T


def test_cut_is_a_balanced_partition():
    S, T = _case()
    g = oracle.build(3, S, T, 40)
    so, _ = g.src_csr()
    to, ti = g.tgt_csr()
    cost = shard_ref.target_costs(T.shape[0], so, to, ti)
    for world in (1, 2, 3, 8):
        ranks = shard_ref.shard_ranks(T, S, 3, so, to, ti, world)
        assert ranks.min() >= 0 and ranks.max() < world
        # Contiguous in the Morton order, ranks ascending along it.
        lo, hi = S.min(axis=0), S.max(axis=0)
        order = np.argsort(shard_ref.morton_keys(T, lo, hi, 3), kind="stable")
        assert np.all(np.diff(ranks[order]) >= 0)
        # Each shard's cost is within one target's cost of total / world.
        per = np.array([cost[ranks == r].sum() for r in range(world)], dtype=np.float64)
        assert per.sum() == float(cost.sum())
        assert np.all(np.abs(per - per.sum() / world) <= float(cost.max()) + 1.0)


def _worker(rank, world, port, S, T, ref, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = oracle.build(3, S, T, 40)
        so, _ = g.src_csr()
        to, ti = g.tgt_csr()
        ranks = shard_ref.shard_ranks(T, S, 3, so, to, ti, world)
        part = np.where(ranks == rank, ref, 0.0)
        pdist.assemble(part)  # numpy, in place
        tpart = torch.from_numpy(np.where(ranks == rank, ref, 0.0))
        pdist.assemble(tpart)  # torch tensor
        q.put((rank, bool(np.array_equal(part, ref)), bool(np.array_equal(tpart.numpy(), ref))))
    finally:
        dist.destroy_process_group()


def test_sharded_outputs_assemble_exactly_over_gloo():
    S, T = _case()
    ref = oracle.interpolate(3, 0x11, S, W.franke_3d(S), T, 40)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, 29511
    procs = [ctx.Process(target=_worker, args=(r, world, port, S, T, ref, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert all(p.exitcode == 0 for p in procs)
    assert res == [(0, True, True), (1, True, True)]


class _OraclePlan:
    """Stand-in for pacman_b200.rbf.Plan on the CPU: the oracle's transfer,
    restricted to the shard that tests/shard_ref.py cuts."""

    def __init__(self, dim, S, T, nodes_per_cluster=50, **_):
        self.dim, self.S, self.T, self.npc = dim, S, T, nodes_per_cluster
        self.owned = None

    def shard(self, rank, world):
        g = oracle.build(self.dim, self.S, self.T, self.npc)
        so, _ = g.src_csr()
        to, ti = g.tgt_csr()
        ranks = shard_ref.shard_ranks(self.T, self.S, self.dim, so, to, ti, world)
        self.owned = ranks == rank
        return self

    def execute(self, basis, values, stats=None):
        out = oracle.interpolate(self.dim, basis, self.S, values, self.T, self.npc)
        return out if self.owned is None else np.where(self.owned, out, 0.0)

    def close(self):
        pass


def _sharded_worker(rank, world, port, S, T, v, ref, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pacman_b200 import rbf as prbf
        prbf.Plan = _OraclePlan  # the wrapper's control flow over the oracle
        full = pdist.interpolate_sharded(3, 0x11, S, v, T, nodes_per_cluster=40)
        part = pdist.interpolate_sharded(3, 0x11, S, v, T, nodes_per_cluster=40, gather=False)
        q.put((rank, bool(np.array_equal(full, ref)), int(np.count_nonzero(part))))
    finally:
        dist.destroy_process_group()


def test_interpolate_sharded_control_flow_over_gloo():
    S, T = _case()
    v = W.franke_3d(S)
    ref = oracle.interpolate(3, 0x11, S, v, T, 40)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, 29512
    procs = [ctx.Process(target=_sharded_worker, args=(r, world, port, S, T, v, ref, q))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert all(p.exitcode == 0 for p in procs)
    assert [r[1] for r in res] == [True, True]
    assert sum(r[2] for r in res) == np.count_nonzero(ref)  # each target on one rank
