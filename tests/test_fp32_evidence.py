"""Why precision "mixed" does not factor in FP32 (CPU only, numpy/LAPACK).

An FP32 Cholesky factor with FP64-residual iterative refinement converges
only while cond(A) * u32 stays moderate.  The patch matrices of the
grid_blobs workload (Wendland C4, support 0.1; here its 10k-point scaled
version, which keeps the full workload's patch sizes and conditioning: the
largest patches hold ~1,700 sources, cond ~1e11) split in two:
* patches of up to 256 sources (cond up to ~5e8): FP32 Cholesky succeeds and
  refinement brings the local values to FP64 accuracy;
* the largest patches: FP32 Cholesky breaks down (a non-positive pivot), and
  refinement with a diagonally shifted FP32 factor does not reach the
  transfer's 1e-10 bound.
The large patches carry almost all of the arithmetic, so the mixed path
emulates FP64 products on the int8 tensor cores for them instead."""
import numpy as np
import pytest
import scipy.linalg as sla

import oracle
from pacman_b200 import workloads as W


def _wendland_c4(r):
    r = np.minimum(r, 1.0)
    return (1.0 - r) ** 6 * (35.0 * r * r + 18.0 * r + 3.0)


@pytest.fixture(scope="module")
def patches():
    w = W.make("grid_blobs_1m", scale=0.01)
    p = oracle.build(3, w["src"], w["tgt"], 50)
    so, si = p.src_csr()
    to, ti = p.tgt_csr()
    return w, so, si, to, ti


def _system(w, so, si, to, ti, k):
    X = w["src"][si[so[k]:so[k + 1]]]
    Y = w["tgt"][ti[to[k]:to[k + 1]]]
    A = _wendland_c4(np.sqrt(((X[:, None] - X[None]) ** 2).sum(-1)) / 0.1)
    E = _wendland_c4(np.sqrt(((Y[:, None] - X[None]) ** 2).sum(-1)) / 0.1)
    return A, E, w["values"][si[so[k]:so[k + 1]], 0]


def _refine(A, L, b, iters):
    x = np.zeros_like(b)
    for _ in range(iters):
        r = b - A @ x
        if not np.all(np.isfinite(r)):
            return None
        x = x + sla.cho_solve((L, True), r.astype(np.float32)).astype(np.float64)
    return x


def test_fp32_refinement_converges_on_patches_up_to_256(patches):
    w, so, si, to, ti = patches
    n, m = np.diff(so), np.diff(to)
    ids = np.where((n > 64) & (n <= 256) & (m > 0))[0]
    rng = np.random.default_rng(0)
    for k in rng.choice(ids, size=min(10, len(ids)), replace=False):
        A, E, b = _system(w, so, si, to, ti, k)
        L = np.linalg.cholesky(A.astype(np.float32))
        x = _refine(A, L, b, 50)
        ref = E @ np.linalg.solve(A, b)
        assert x is not None
        assert np.linalg.norm(E @ x - ref) / np.linalg.norm(ref) < 1e-12


def test_fp32_breaks_down_on_the_largest_patches(patches):
    w, so, si, to, ti = patches
    n = np.diff(so)
    for k in np.argsort(-n)[:3]:
        assert n[k] > 1000
        A, E, b = _system(w, so, si, to, ti, k)
        with pytest.raises(np.linalg.LinAlgError):
            np.linalg.cholesky(A.astype(np.float32))
        shift = 1e-6 * np.abs(A).max() * np.sqrt(len(b))
        L = np.linalg.cholesky((A + shift * np.eye(len(b))).astype(np.float32))
        x = _refine(A, L, b, 50)
        ref = E @ np.linalg.solve(A, b)
        err = np.inf if x is None else np.linalg.norm(E @ x - ref) / np.linalg.norm(ref)
        assert not err <= 1e-10, (k, n[k], err)
