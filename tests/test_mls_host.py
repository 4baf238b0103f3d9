"""Moving least squares: the CPU oracle and the host side of pacman.MLS.

The reference computes MLS with ArborX 2.1's MovingLeastSquares (an
un-vendored dependency, src/mls/interpolator.hpp:49-77), so the oracle
restates that published algorithm (oracle/rbf_pum_oracle.c,
orc_mls_interpolate) and is pinned here by
* the reference's own MLS known answers: tests/test_mls.py:83-92 (20^D grid
  onto itself in 1D, 2D, 3D, Franke, rel-L2 < 1e-4) and
  tests/test_cpp_mls_interface.cpp:148-151 (the 3D case through the C++ API);
* an independent numpy statement of the same fit (LAPACK pseudo-inverse of
  the moment matrix instead of the oracle's Jacobi rotations);
* exact reproduction of quadratic polynomials, which a degree-2 MLS fit has
  whenever its moment matrix is invertible.
With as many neighbours as basis functions the fit is an interpolation whose
moment matrix can be close to singular (cond(A) up to ~1e11 on random 3D
clouds); two FP64 evaluations then agree to rounding x cond(A), and the
comparisons scale their bound by each target's cond(A).  The CUDA kernel
is compared with the oracle bit for bit (tests/test_gpu_mls.py)."""
import numpy as np
import pytest

import oracle
import pacman
from pacman_b200 import workloads as W

K = {1: 3, 2: 6, 3: 10}


def _grid(n, dim):
    axes = np.meshgrid(*([np.linspace(0.0, 1.0, n)] * dim), indexing="ij")
    return np.stack([a.ravel() for a in axes], axis=1)


def _basis(x):
    if len(x) == 1:
        return np.array([1.0, x[0], x[0] ** 2])
    if len(x) == 2:
        return np.array([1.0, x[0], x[1], x[0] ** 2, x[0] * x[1], x[1] ** 2])
    return np.array([1.0, *x, x[0] ** 2, x[0] * x[1], x[0] * x[2], x[1] ** 2, x[1] * x[2],
                     x[2] ** 2])


def _mls_numpy(S, f, T, with_cond=False):
    """The same fit with LAPACK's pseudo-inverse; with_cond adds cond(A) per
    target (the value's sensitivity to rounding grows with it)."""
    k = min(K[S.shape[1]], len(S))
    out = np.zeros(len(T))
    cond = np.zeros(len(T))
    for i, t in enumerate(T):
        d2 = ((S - t) ** 2).sum(1)
        idx = np.lexsort((np.arange(len(S)), d2))[:k]
        d = np.sqrt(d2[idx])
        r = 1.1 * max(10 * np.finfo(float).eps, d.max())
        w = (1.0 - d / r) ** 2
        P = np.array([_basis(x) for x in (S[idx] - t) / r])
        A = P.T @ (w[:, None] * P)
        out[i] = (np.linalg.pinv(A, rcond=1e-13, hermitian=True) @ (P.T @ (w * f[idx])))[0]
        lam = np.abs(np.linalg.eigvalsh(A))
        cond[i] = lam.max() / max(lam.min(), 1e-300)
    return (out, cond) if with_cond else out


def _agree(out, ref, cond):
    """Two FP64 evaluations of one fit agree to rounding x cond(A)."""
    bound = 1e-14 * np.minimum(cond, 1e12) * np.maximum(1.0, np.abs(ref)) + 1e-13
    assert (np.abs(out - ref) <= bound).all(), np.max(np.abs(out - ref) / bound)
    assert np.median(np.abs(out - ref)) < 1e-13


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_reference_grid_known_answer(dim):
    g = _grid(20, dim)
    v = W.franke(g)
    out = oracle.mls_interpolate(dim, g, v, g)
    assert np.linalg.norm(out - v) / np.linalg.norm(v) < 1e-4


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_oracle_matches_numpy_pseudo_inverse(dim):
    rng = np.random.default_rng(10 + dim)
    S = rng.random((1500, dim))
    T = rng.random((300, dim))
    f = W.franke(S)
    out, sweeps = oracle.mls_interpolate(dim, S, f, T, with_sweeps=True)
    ref, cond = _mls_numpy(S, f, T, with_cond=True)
    _agree(out, ref, cond)
    assert sweeps.max() < 16


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_quadratics_are_reproduced(dim):
    rng = np.random.default_rng(20 + dim)
    n = {1: 200, 2: 30, 3: 12}[dim]
    S = (_grid(n, dim) + rng.uniform(-0.3, 0.3, size=(n ** dim, dim)) / n)
    T = rng.random((400, dim))
    q = lambda p: 1.0 + p.sum(1) - 2.0 * (p ** 2).sum(1) + 3.0 * p[:, 0] * p[:, -1]  # noqa: E731
    out = oracle.mls_interpolate(dim, S, q(S), T)
    _, cond = _mls_numpy(S, q(S), T, with_cond=True)
    _agree(out, q(T), cond)


def _neighbour_cases():
    rng = np.random.default_rng(50)
    cases = []
    for dim in (1, 2, 3):
        S = rng.random((6000, dim))
        cases.append((dim, S, W.franke(S), rng.random((2000, dim))))
    g = _grid(20, 3)
    cases.append((3, g, W.franke(g), g))                       # exact distance ties
    c = rng.random((8, 3))
    S = c[rng.integers(0, 8, 20000)] + rng.normal(0.0, 0.02, size=(20000, 3))
    T = np.concatenate([rng.random((2000, 3)), rng.random((200, 3)) * 4.0 + 2.0])
    cases.append((3, S, S[:, 0], T))                           # clusters, far targets
    b = rng.random((1500, 3))
    S = np.concatenate([b, b[:700]])
    cases.append((3, S, rng.standard_normal(len(S)), rng.random((1500, 3))))  # duplicates
    P = np.c_[rng.random((3000, 2)), np.zeros(3000)]
    cases.append((3, P, W.franke(P), np.c_[rng.random((1000, 2)), rng.choice([0.0, 0.05], 1000)]))
    return cases


def test_grid_neighbour_search_equals_brute_force():
    """The oracle's cell-grid neighbour search (used from 4,096 sources on)
    finds the same neighbours in the same order as the all-pairs scan, so the
    values are identical."""
    for dim, S, f, T in _neighbour_cases():
        a = oracle.mls_interpolate(dim, S, f, T, knn="brute")
        b = oracle.mls_interpolate(dim, S, f, T, knn="grid")
        assert np.array_equal(a, b), (dim, len(S))


def test_fewer_sources_than_the_basis_and_none():
    rng = np.random.default_rng(3)
    T = rng.random((50, 3))
    # One source: the pseudo-inverse fit of one value.
    S = np.array([[0.5, 0.5, 0.5]])
    out = oracle.mls_interpolate(3, S, np.array([2.0]), T)
    assert np.allclose(out, _mls_numpy(S, np.array([2.0]), T), rtol=1e-12, atol=1e-14)
    S = rng.random((4, 3))
    f = rng.random(4)
    assert np.allclose(oracle.mls_interpolate(3, S, f, T), _mls_numpy(S, f, T), rtol=1e-9,
                       atol=1e-12)
    assert (oracle.mls_interpolate(3, np.zeros((0, 3)), np.zeros(0), T) == 0).all()


@pytest.mark.parametrize("sp,sv,tp,exc", [
    (np.zeros(5), np.zeros(5), np.zeros((4, 3)), ValueError),
    (np.zeros((5, 3)), np.zeros(5), np.zeros(4), ValueError),
    (np.zeros((5, 3)), np.zeros(5), np.zeros((4, 2)), ValueError),
    (np.zeros((5, 3)), np.zeros(4), np.zeros((4, 3)), ValueError),
])
def test_python_argument_checks(sp, sv, tp, exc):
    """mls_bindings.cpp: the binding's shape checks, before any device work."""
    with pytest.raises(exc):
        pacman.MLS.interpolate(3, pacman.execspaces.CUDA, sp, sv, tp)


def test_python_dimension_and_empty_targets():
    with pytest.raises(RuntimeError, match="1, 2 or 3"):
        pacman.MLS.interpolate(4, 3, np.zeros((5, 4)), np.zeros(5), np.zeros((2, 4)))
    out = pacman.MLS.interpolate(3, 3, np.zeros((5, 3)), np.zeros(5), np.zeros((0, 3)))
    assert out.shape == (0,)


def test_kernel_is_built_without_contraction():
    """The GPU values equal the oracle's bit for bit only while mls.cu is
    compiled without fused multiply-adds (the oracle uses -ffp-contract=off)."""
    from pacman_b200 import build
    assert "-fmad=false" in build.FILE_FLAGS["mls.cu"]
    import os
    mk = open(os.path.join(os.path.dirname(oracle.__file__), "Makefile")).read()
    assert "-ffp-contract=off" in mk
