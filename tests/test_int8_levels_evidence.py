"""Why the int8 column updates keep the digit levels a + b <= 9 (CPU only).

Precision "mixed" stores every off-diagonal Cholesky tile L[i, p] as 7 int8
digits of L / sigma and forms the column updates sum_p L[i, p] L[j, p]^T from
the digit products of level a + b <= 9 (pacman_b200/csrc/cholesky.cu,
slice_tile_smem and the k_col_step_ws MMA schedule; sigma and the digit
multiplier in pacman_b200/csrc/blocked.cu).  This file models that
factorisation on the CPU with exact digit products (integer-valued FP64
matrix products, exact below 2^53) and the same 64-wide left-looking tile
order, on sampled patches of the shell workload (4M sources on a perturbed
sphere shell plus the enclosing cube, Wendland C4, patches of 512-1,024
sources, cond(A) 1e11-1e14), and compares the local values with those of
LAPACK's LU:
* with levels <= 9 the error is that of the same factorisation with FP64
  column updates;
* with levels <= 8 it grows several-fold on most patches, so level 9 is the
  cheapest cut that leaves the transfer at FP64 accuracy."""
import numpy as np
import pytest
import scipy.linalg as sla

import oracle
from pacman_b200 import workloads as W

SLICES = 7
TB = 64
# sigma >= sqrt(phi(0)) bounds every |L| (rows of L have norm sqrt(A_rr));
# Wendland C4 has phi(0) = 3.
SIGMA = np.sqrt(3.0) * (128.0 / 127.0) * (1.0 + 2.0 ** -20)


def _wendland_c4(p):
    p = np.minimum(p, 1.0)
    return (1.0 - p) ** 6 * (35.0 * p * p + 18.0 * p + 3.0)


def _digits(Lt):
    """The 7 balanced base-128 digits of Lt / SIGMA, most significant first:
    y = round(x 128^7); d = round(y / 128^(6 - s)), y -= d 128^(6 - s)."""
    xs = np.clip(Lt * (128.0 / SIGMA), -127.49, 127.49)
    y = np.rint(xs * 2.0 ** 42).astype(np.int64)
    out = []
    for s in range(SLICES):
        sh = 7 * (SLICES - 1 - s)
        d = ((y + (1 << (sh - 1))) >> sh) if sh else y.copy()
        y = y - (d << sh)
        out.append(d)
    return out


def _cholesky(A, max_level):
    """Left-looking 64-wide tiled Cholesky of A (padded with the identity).
    Diagonal tiles are updated in FP64; the off-diagonal column updates use
    the digit products of level <= max_level (None: FP64 products)."""
    n0 = len(A)
    T = -(-n0 // TB)
    N = T * TB
    Ap = np.eye(N)
    Ap[:n0, :n0] = A
    L = np.zeros((N, N))
    D = [np.zeros((N, N)) for _ in range(SLICES)]
    for j in range(T):
        cj, K, rest = slice(j * TB, (j + 1) * TB), j * TB, slice((j + 1) * TB, N)
        L[cj, cj] = np.linalg.cholesky(Ap[cj, cj] - L[cj, :K] @ L[cj, :K].T)
        if j == T - 1:
            break
        if max_level is None:
            C = Ap[rest, cj] - L[rest, :K] @ L[cj, :K].T
        else:
            acc = np.zeros(((T - j - 1) * TB, TB))
            for s in range(2, max_level + 1):
                level = np.zeros_like(acc)
                for a in range(max(1, s - SLICES), min(SLICES, s - 1) + 1):
                    level += D[a - 1][rest, :K] @ D[s - a - 1][cj, :K].T
                acc += level * 2.0 ** (-7 * s)
            C = Ap[rest, cj] - SIGMA * SIGMA * acc
        L[rest, cj] = sla.solve_triangular(L[cj, cj], C.T, lower=True).T
        for q, d in enumerate(_digits(L[rest, cj])):
            D[q][rest, cj] = d
    return L[:n0, :n0]


def test_digits_reconstruct_the_factor_to_49_bits():
    rng = np.random.default_rng(5)
    x = rng.uniform(-1.0, 1.0, size=(64, 64)) * SIGMA * (127.0 / 128.0)
    d = _digits(x)
    assert np.abs(d[0]).max() <= 127
    assert all(np.abs(di).max() <= 64 for di in d[1:])
    back = sum(di.astype(np.float64) * 128.0 ** -(s + 1) for s, di in enumerate(d))
    assert np.abs(back * SIGMA - x).max() <= SIGMA * 2.0 ** -49


@pytest.fixture(scope="module")
def shell_errors():
    S = W._shell_cube(4_000_000, 21)
    Tg = W._shell_cube(2_000_000, 22)
    p = oracle.build(3, S, Tg, 50)
    so, si = p.src_csr()
    to, ti = p.tgt_csr()
    n, m = np.diff(so), np.diff(to)
    rng = np.random.default_rng(0)
    ids = rng.choice(np.where((n > 512) & (n <= 1024) & (m > 0))[0], size=8, replace=False)
    rows = []
    for k in ids:
        X = S[si[so[k]:so[k + 1]]]
        Y = Tg[ti[to[k]:to[k + 1]]]
        b = W.franke_3d(X)
        A = _wendland_c4(np.sqrt(((X[:, None] - X[None]) ** 2).sum(-1)) / 0.1)
        E = _wendland_c4(np.sqrt(((Y[:, None] - X[None]) ** 2).sum(-1)) / 0.1)
        Q, Vm = np.c_[np.ones(len(X)), X], np.c_[np.ones(len(Y)), Y]
        beta = np.linalg.lstsq(Q, b, rcond=None)[0]
        r = b - Q @ beta
        ref = E @ np.linalg.solve(A, r) + Vm @ beta
        err = {}
        for cut in (None, 8, 9):
            v = E @ sla.cho_solve((_cholesky(A, cut), True), r) + Vm @ beta
            err[cut] = np.linalg.norm(v - ref) / np.linalg.norm(ref)
        rows.append((int(k), len(X), err))
    return rows


def test_level_9_matches_fp64_updates(shell_errors):
    for k, n, err in shell_errors:
        assert err[9] <= 2.0 * err[None] + 1e-15, (k, n, err)


def test_level_8_is_not_enough(shell_errors):
    ratios = sorted(err[8] / err[9] for _, _, err in shell_errors)
    assert all(r > 1.5 for r in ratios), ratios
    assert ratios[len(ratios) // 2] > 4.0, ratios
