"""Kept factorisations (PACMAN_B200_KEEP_FACTORS, ``Plan.execute(keep_factors=True)``).

The factorising execute must give exactly what an execute without the flag
gives; a later execute with new values reuses the factors (only the
polynomial block, the triangular solves and the evaluation run) and must
match a fresh transfer of those values: within 1e-12 relative L2 (the forward
substitution of the large patches runs in another order) and within the
mixed path's 1e-10 of the CPU oracle."""
import numpy as np
import pytest

import oracle
import pacman_b200 as pacman
from pacman_b200 import workloads as W
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_REUSE = 1e-12
TOL_MIXED = 1e-10


def _cases():
    rng = np.random.default_rng(12)
    gb = W.make("grid_blobs_1m", scale=0.01)
    u = W.make("uniform_20k", scale=0.5)
    S2, T2 = rng.random((6000, 2)), rng.random((5000, 2))
    return {
        "grid_blobs_10k_c4": (3, gb["src"], gb["tgt"], 0x12, 50),
        "uniform_10k_c2": (3, u["src"], u["tgt"], 0x11, 30),
        "uniform_2d_c6": (2, S2, T2, 0x13, 40),
    }


CASES = _cases()


def _fields(S, F, seed):
    rng = np.random.default_rng(seed)
    k = rng.uniform(1.0, 4.0, size=(F, S.shape[1]))
    v = np.stack([np.sin(S @ k[f]) + 0.3 * f for f in range(F)], axis=1)
    return v[:, 0] if F == 1 else v


def _solved_patches(plan):
    off, _ = plan.patch_lists("target")
    return int(np.count_nonzero(np.diff(off)))


@pytest.mark.parametrize("name", sorted(CASES))
def test_reuse_matches_fresh_transfers(name):
    dim, S, T, basis, npc = CASES[name]
    plan = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="mixed")
    v1, v2, v3 = _fields(S, 1, 1), _fields(S, 3, 2), _fields(S, 2, 3)
    st = {}
    out1 = plan.execute(basis, v1, stats=st, keep_factors=True)
    assert st["factors_reused"] == 0
    fresh = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="mixed")
    assert np.array_equal(out1, fresh.execute(basis, v1))
    nsolved = _solved_patches(plan)
    for v in (v2, v3, v1):
        st = {}
        out = plan.execute(basis, v, stats=st, keep_factors=True)
        assert st["factors_reused"] == nsolved
        ref = fresh.execute(basis, v)
        assert out.shape == ref.shape
        assert rel_l2(out, ref) <= TOL_REUSE
    ora = oracle.interpolate(dim, basis, S, v2, T, npc)
    out2 = plan.execute(basis, v2, keep_factors=True)
    assert rel_l2(out2, ora) <= TOL_MIXED
    # Without the flag the plan factors afresh and leaves the kept factors.
    assert np.array_equal(plan.execute(basis, v2), fresh.execute(basis, v2))
    st = {}
    plan.execute(basis, v3, stats=st, keep_factors=True)
    assert st["factors_reused"] == nsolved
    plan.close()
    fresh.close()


def test_basis_change_refactors():
    dim, S, T, basis, npc = CASES["grid_blobs_10k_c4"]
    v = _fields(S, 1, 4)
    plan = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="mixed")
    plan.execute(basis, v, keep_factors=True)
    st = {}
    out = plan.execute(0x13, v, stats=st, keep_factors=True)
    assert st["factors_reused"] == 0
    fresh = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="mixed")
    assert np.array_equal(out, fresh.execute(0x13, v))
    st = {}
    out = plan.execute(0x13, v, stats=st, keep_factors=True)
    assert st["factors_reused"] > 0
    assert rel_l2(out, fresh.execute(0x13, v)) <= TOL_REUSE


def test_fp64_and_shard_keep_nothing():
    dim, S, T, basis, npc = CASES["uniform_2d_c6"]
    v = _fields(S, 1, 5)
    plan = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="fp64")
    ref = plan.execute(basis, v)
    for _ in range(2):
        st = {}
        assert np.array_equal(plan.execute(basis, v, stats=st, keep_factors=True), ref)
        assert st["factors_reused"] == 0
    plan.close()
    plan = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="mixed")
    plan.execute(basis, v, keep_factors=True)
    plan.shard(0, 2)
    st = {}
    plan.execute(basis, v, stats=st, keep_factors=True)
    assert st["factors_reused"] == 0
    st = {}
    plan.execute(basis, v, stats=st, keep_factors=True)
    assert st["factors_reused"] > 0


def test_reuse_with_adjoint():
    dim, S, T, basis, npc = CASES["grid_blobs_10k_c4"]
    v = _fields(S, 2, 6)
    g = np.random.default_rng(7).standard_normal((T.shape[0], 2))
    plan = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="mixed")
    plan.execute(basis, v, keep_factors=True)
    st = {}
    out = plan.execute(basis, v, keep_factors=True, save_for_adjoint=True, stats=st)
    assert st["factors_reused"] > 0 and st["patches_fallback"] == 0
    gv, gt = plan.adjoint(g)
    fresh = pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc, precision="mixed")
    st = {}
    out0 = fresh.execute(basis, v, save_for_adjoint=True, stats=st)
    assert st["patches_fallback"] == 0
    assert rel_l2(out, out0) <= TOL_REUSE
    assert rel_l2(plan.local_values(), fresh.local_values()) <= TOL_REUSE
    gv0, gt0 = fresh.adjoint(g)
    assert rel_l2(gv, gv0) <= 1e-11
    assert rel_l2(gt, gt0) <= 1e-11
