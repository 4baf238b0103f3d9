"""The CPU oracle against the reference's own known-answer tests, and its
grid search against brute force.  CPU only."""
import numpy as np
import pytest

import oracle
from pacman_b200 import workloads as W
from tests.conftest import grid_cloud, rel_l2, slab_meshes

BASES = [0x10, 0x11, 0x12, 0x13, 0x14]


@pytest.mark.parametrize("basis", BASES)
def test_grid20_node_reproduction(basis):
    # tests/test_cpp_rbf_interface.cpp:165-198: same -> same, rel-L2 < 1e-8.
    P = grid_cloud(20)
    v = W.franke_3d(P)
    out = oracle.interpolate(3, basis, P, v, P)
    assert rel_l2(out, v) < 1e-8


@pytest.mark.parametrize("pair", [("0.03", "0.003"), ("0.003", "0.03"), ("0.03", "0.03")])
@pytest.mark.parametrize("basis", BASES)
def test_slab_meshes_franke(pair, basis):
    # tests/test_rbf-pum.py:58-74: every file name holds a '3', so tol 1.5e-2.
    m = slab_meshes()
    S, T = m[pair[0]], m[pair[1]]
    out = oracle.interpolate(3, basis, S, W.franke_3d(S), T)
    assert rel_l2(out, W.franke_3d(T)) < 1.5e-2


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("n,m", [(2500, 1800), (400, 700)])
def test_grid_search_equals_brute_force(dim, n, m):
    rng = np.random.default_rng(100 * dim + n)
    S = rng.random((n, dim))
    T = rng.random((m, dim)) * 1.3 - 0.15
    a = oracle.build(dim, S, T, 30)
    b = oracle.build(dim, S, T, 30, brute_force=True)
    assert a.radius == b.radius
    assert a.num_patches == b.num_patches
    assert np.array_equal(a.centers(), b.centers())
    for x, y in zip(a.src_csr(), b.src_csr()):
        assert np.array_equal(x, y)
    for x, y in zip(a.tgt_csr(), b.tgt_csr()):
        assert np.array_equal(x, y)
    assert np.array_equal(a.weight_sums(), b.weight_sums())


def test_partition_of_unity_and_linear_reproduction():
    # The normalised weights of a target covered by patches sum to one, so a
    # linear field (reproduced exactly by every local interpolant thanks to
    # the polynomial block) comes back to rounding level.
    rng = np.random.default_rng(7)
    S = rng.random((3000, 3))
    T = rng.random((2000, 3)) * 0.9 + 0.05
    lin = 0.3 + S @ np.array([1.0, -2.0, 0.5])
    out = oracle.interpolate(3, 0x11, S, lin, T, 30)
    ref = 0.3 + T @ np.array([1.0, -2.0, 0.5])
    assert rel_l2(out, ref) < 1e-10


def test_multifield_equals_single_fields():
    rng = np.random.default_rng(8)
    S = rng.random((1500, 3))
    T = rng.random((1200, 3))
    V = np.stack([W.franke_3d(S), np.sin(3 * S[:, 0]), S[:, 1] ** 2], axis=1)
    plan = oracle.build(3, S, T, 30)
    multi, _, _ = plan.solve(0x12, V)
    for f in range(3):
        single, _, _ = plan.solve(0x12, V[:, f])
        assert np.array_equal(multi[:, f], single)


def test_degenerate_planar_patches_drop_an_axis():
    # 3D points on the plane z = 0.5: every patch's [1, x, y, z] block is
    # rank deficient, so the condition loop drops the z axis.
    rng = np.random.default_rng(9)
    S = np.c_[rng.random((2000, 2)), np.full(2000, 0.5)]
    T = np.c_[rng.random((1000, 2)), np.full(1000, 0.5)]
    f = lambda P: np.cos(2 * P[:, 0]) + P[:, 1]
    plan = oracle.build(3, S, T, 30)
    out, _, st = plan.solve(0x11, f(S))
    assert st["dropped_axis_patches"] == plan.num_patches
    assert rel_l2(out, f(T)) < 1e-3


@pytest.mark.parametrize("dim,N", [(1, 400), (2, 40)])
def test_node_reproduction_1d_2d(dim, N):
    # The 20^3 known answer of tests/test_cpp_rbf_interface.cpp:165-198 in one
    # and two dimensions: a regular grid transferred onto itself reproduces
    # the source values (rel-L2 < 1e-8, every basis).
    g = np.arange(N) / (N - 1.0)
    P = np.stack(np.meshgrid(*([g] * dim), indexing="ij"), axis=-1).reshape(-1, dim)
    v = np.cos(3 * P[:, 0]) + (P[:, 1] ** 2 if dim > 1 else 0.0)
    for basis in BASES:
        out = oracle.interpolate(dim, basis, P, v, P, 30)
        assert rel_l2(out, v) < 1e-8, basis


def test_weights_sum_to_one_and_locals_interpolate_the_nodes():
    # Every target inside the cover has normalised partition-of-unity weights
    # summing to one (the un-normalised sums are positive), and every local
    # interpolant reproduces the source values at its own nodes (targets equal
    # to sources, so each patch's target list holds its interior nodes).
    rng = np.random.default_rng(10)
    S = rng.random((2500, 3))
    v = W.franke_3d(S)
    plan = oracle.build(3, S, S, 30)
    assert (plan.weight_sums() > 0).all()
    ones, _, _ = plan.solve(0x11, np.ones(len(S)))
    assert np.max(np.abs(ones - 1.0)) < 1e-12
    _, local, _ = plan.solve(0x11, v, want_local=True)
    toff, tidx = plan.tgt_csr()
    assert rel_l2(local[:, 0] if local.ndim == 2 else local, v[tidx]) < 1e-12
