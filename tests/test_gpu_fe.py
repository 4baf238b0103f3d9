"""NEAREST_NEAREST finite-element transfer on the GPU (pacman_b200.fe through
pacman_b200_fe_interpolate) against the CPU oracle: the chosen source must be
the oracle's exactly (random source values, so equal values mean equal
sources), the status OUTSIDE (0) everywhere as in the reference."""
import numpy as np
import pytest

import oracle
import pacman_b200 as pacman

pytestmark = pytest.mark.gpu

FE = pacman.fe
NN = FE.methods.NEAREST_NEAREST


def _check(dim, S, T, seed=0):
    v = np.random.default_rng(seed).standard_normal(S.shape[0])
    out, status = FE.interpolate(dim, pacman.execspaces.CUDA, NN, S, v, None, None, None, T)
    ref, _ = oracle.fe_nearest(dim, S, v, T)
    assert np.array_equal(out, ref)
    assert status.dtype == np.int32 and np.all(status == 0)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_uniform_and_outside(dim):
    rng = np.random.default_rng(10 + dim)
    S = rng.random((20000, dim))
    T = rng.uniform(-0.2, 1.2, size=(15000, dim))  # some targets outside the sources' box
    _check(dim, S, T)


def test_clustered_and_far_targets():
    rng = np.random.default_rng(4)
    S = np.concatenate([rng.random((5000, 3)), 0.3 + 0.01 * rng.standard_normal((20000, 3))])
    T = np.concatenate([rng.random((8000, 3)), rng.random((50, 3)) * 100.0 + 50.0])
    _check(3, S, T, 1)


def test_identity_ties_and_degenerate():
    rng = np.random.default_rng(5)
    S = rng.random((3000, 3))
    _check(3, S, S, 2)                                 # the reference's known answer
    D = np.concatenate([S, S, S[:100]])                # exact duplicates: lowest index wins
    _check(3, D, rng.random((2000, 3)), 3)
    G = np.stack(np.meshgrid(np.arange(8.0), np.arange(8.0), indexing="ij"), -1).reshape(-1, 2)
    _check(2, G, G + 0.5, 4)                           # four equidistant sources per target
    P = np.c_[rng.random((4000, 2)), np.zeros(4000)]   # planar sources in 3D
    _check(3, P, rng.random((1000, 3)), 5)
    _check(3, S[:1], rng.random((100, 3)), 6)          # one source


def test_no_sources_and_device_tensors():
    T = np.random.default_rng(6).random((100, 3))
    out, status = FE.interpolate(3, 3, NN, np.zeros((0, 3)), np.zeros(0), None, None, None, T)
    assert np.all(out == 0.0) and np.all(status == 0)
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    S, T = rng.random((5000, 3)), rng.random((4000, 3))
    v = rng.standard_normal(5000)
    out, status = FE.interpolate(3, 3, NN, torch.tensor(S, device="cuda"),
                                 torch.tensor(v, device="cuda"), None, None, None,
                                 torch.tensor(T, device="cuda"))
    assert out.is_cuda and status.is_cuda
    ref, _ = oracle.fe_nearest(3, S, v, T)
    assert np.array_equal(out.cpu().numpy(), ref)
    assert int(status.abs().sum()) == 0
    with pytest.raises(ValueError):
        FE.interpolate(3, 3, FE.methods.INTERP_CLAMP, S, v, None, None, None, T)
