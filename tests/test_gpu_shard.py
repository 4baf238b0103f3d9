"""Target sharding on one GPU: the ranks of a sharded transfer run one after
another (each its own plan; nothing waits on another rank), and

* the owned target sets are the CPU restatement's cut (tests/shard_ref.py),
  disjoint and covering;
* the sum of the ranks' outputs is bit-identical to the unsharded transfer;
* the ranks' adjoint contributions sum to the unsharded adjoint."""
import numpy as np
import pytest

import pacman_b200 as pacman
from pacman_b200 import workloads as W
from tests import shard_ref
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(8)
    gb = W.make("grid_blobs_1m", scale=0.01)
    S2, T2 = rng.random((6000, 2)), rng.random((5000, 2))
    u = W.make("uniform_20k", scale=0.5)
    return {
        "grid_blobs_10k_c4": (3, gb["src"], gb["tgt"], gb["values"][:, 0], 0x12, 50),
        "uniform_10k_c2_2f": (3, u["src"], u["tgt"],
                              np.c_[u["values"][:, 0], np.sin(3 * u["src"][:, 1])], 0x11, 30),
        "uniform_2d_c6": (2, S2, T2, np.sin(4 * S2[:, 0]) * np.cos(3 * S2[:, 1]), 0x13, 40),
    }


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sharded_sum_is_bit_identical(name, precision):
    dim, S, T, v, basis, npc = CASES[name]
    full = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision=precision)
    ref = full.execute(basis, v)
    so, _ = full.patch_lists("source")
    to, ti = full.patch_lists("target")
    full.close()
    for world in (2, 3, 4):
        want = shard_ref.shard_ranks(T, S, dim, so, to, ti, world)
        total = np.zeros_like(ref)
        seen = np.zeros(T.shape[0], dtype=np.int64)
        for rank in range(world):
            p = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision=precision)
            p.shard(rank, world)
            owned = p.owned_targets()
            assert np.array_equal(owned, np.nonzero(want == rank)[0])
            out = p.execute(basis, v)
            p.close()
            others = np.ones(T.shape[0], dtype=bool)
            others[owned] = False
            assert np.all(out[others] == 0.0)
            total += out
            seen[owned] += 1
        assert np.all(seen == 1)
        assert np.array_equal(total, ref), (world, float(np.abs(total - ref).max()))


def test_sharded_adjoint_sums():
    dim, S, T, v, basis, npc = CASES["uniform_10k_c2_2f"]
    rng = np.random.default_rng(2)
    g = rng.standard_normal((T.shape[0], 2))
    full = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc)
    full.execute(basis, v, save_for_adjoint=True)
    gv_ref, gt_ref = full.adjoint(g)
    full.close()
    world = 3
    gv = np.zeros_like(gv_ref)
    gt = np.zeros_like(gt_ref)
    for rank in range(world):
        p = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc)
        p.shard(rank, world)
        p.execute(basis, v, save_for_adjoint=True)
        a, b = p.adjoint(g)
        p.close()
        gv += a
        gt += b
    assert rel_l2(gv, gv_ref) <= 1e-12
    assert np.array_equal(gt, gt_ref)


def test_shard_errors():
    dim, S, T, v, basis, npc = CASES["uniform_2d_c6"]
    p = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc)
    with pytest.raises(ValueError):
        p.shard(2, 2)
    p.shard(0, 1)
    assert np.array_equal(p.owned_targets(), np.arange(T.shape[0]))
    with pytest.raises(ValueError):
        p.shard(0, 2)  # already sharded
    p.close()
