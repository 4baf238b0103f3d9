"""Seeded synthetic point clouds and fields for the RBF-PUM transfer.

The reference publishes no benchmark data set; these generators produce the
five transfer workloads the project measures (all numpy ``default_rng`` with
fixed seeds, FP64 row-major points):

* ``uniform_20k``            20k -> 20k uniform in [0,1]^3, Wendland C2,
                             30 nodes per cluster, Franke 3D field.
* ``grid_blobs_1m``          1M sources (500k jittered 100^3 grid cells +
                             500k from 64 Gaussian blobs, sigma 0.02) ->
                             1M uniform targets, Wendland C4, Franke 3D.
* ``shell_4m``               4M sources (60% on a perturbed unit sphere shell,
                             40% uniform in [-1.05, 1.05]^3) -> 2M targets
                             drawn the same way, 8 fields.
* ``uniform_500k``           500k -> 500k uniform, Wendland C4, 4 fields.
* ``many_256``               256 independent uneven problems.

``scale`` shrinks a workload's point counts (the sizes the CPU oracle can
check in seconds) while keeping its shape and value distributions.
"""
from __future__ import annotations

import numpy as np

WENDLANDC0, WENDLANDC2, WENDLANDC4, WENDLANDC6, WENDLANDC8 = 0x10, 0x11, 0x12, 0x13, 0x14


def franke_3d(p: np.ndarray) -> np.ndarray:
    """Franke's 3D test function (tests/franke_functions.py:118-166 of the reference)."""
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    return (0.75 * np.exp(-((9 * x - 2) ** 2 + (9 * y - 2) ** 2 + (9 * z - 2) ** 2) / 4.0)
            + 0.75 * np.exp(-((9 * x + 1) ** 2 / 49.0 + (9 * y + 1) / 10.0 + (9 * z + 1) / 10.0))
            + 0.5 * np.exp(-((9 * x - 7) ** 2 + (9 * y - 3) ** 2 + (9 * z - 5) ** 2) / 4.0)
            - 0.2 * np.exp(-((9 * x - 4) ** 2 + (9 * y - 7) ** 2 + (9 * z - 5) ** 2)))


def franke_2d(p: np.ndarray) -> np.ndarray:
    """Franke's 2D test function (tests/franke_functions.py:71-116 of the reference)."""
    x, y = p[:, 0], p[:, 1]
    return (0.75 * np.exp(-((9 * x - 2) ** 2 + (9 * y - 2) ** 2) / 4.0)
            + 0.75 * np.exp(-((9 * x + 1) ** 2 / 49.0 + (9 * y + 1) / 10.0))
            + 0.5 * np.exp(-((9 * x - 7) ** 2 + (9 * y - 3) ** 2) / 4.0)
            - 0.2 * np.exp(-((9 * x - 4) ** 2 + (9 * y - 7) ** 2)))


def franke_1d(p: np.ndarray) -> np.ndarray:
    """The reference's 1D Franke function (tests/franke_functions.py:29-69, the
    later of its two definitions, which is the one Python keeps)."""
    x = p[:, 0]
    return (0.75 * np.exp(-((9 * x - 2) ** 2) / 4.0)
            + 0.75 * np.exp(-((9 * x + 1) ** 2) / 49.0)
            + 0.5 * np.exp(-((9 * x - 7) ** 2) / 4.0)
            - 0.2 * np.exp(-((9 * x - 4) ** 2)))


def franke(p: np.ndarray) -> np.ndarray:
    """franke_1d, franke_2d or franke_3d by the points' dimension."""
    return {1: franke_1d, 2: franke_2d, 3: franke_3d}[p.shape[1]](p)


def fourier_fields(p: np.ndarray, nfields: int, seed: int, modes: int = 16, kmax: int = 4) -> np.ndarray:
    """nfields random Fourier series sum_j a_j cos(2 pi k_j.x) + b_j sin(2 pi k_j.x),
    a, b ~ N(0,1), integer wavenumbers with |k|_inf <= kmax."""
    rng = np.random.default_rng(seed)
    out = np.empty((p.shape[0], nfields))
    for f in range(nfields):
        k = rng.integers(-kmax, kmax + 1, size=(modes, 3))
        a = rng.standard_normal(modes)
        b = rng.standard_normal(modes)
        ph = 2.0 * np.pi * (p @ k.T.astype(np.float64))
        out[:, f] = np.cos(ph) @ a + np.sin(ph) @ b
    return out


def _uniform(n, seed, lo=0.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=(n, 3))


def _grid_blobs(n, seed):
    rng = np.random.default_rng(seed)
    n_grid = n // 2
    n_blob = n - n_grid
    cells = rng.choice(100 ** 3, size=n_grid, replace=False)
    ijk = np.stack(np.unravel_index(cells, (100, 100, 100)), axis=1).astype(np.float64)
    grid = (ijk + 0.5) / 100.0 + rng.uniform(-0.3, 0.3, size=(n_grid, 3)) / 100.0
    centres = rng.uniform(0.0, 1.0, size=(64, 3))
    which = rng.integers(0, 64, size=n_blob)
    blobs = centres[which] + rng.normal(0.0, 0.02, size=(n_blob, 3))
    pts = np.concatenate([grid, blobs])
    return pts[rng.permutation(n)]


def _shell_cube(n, seed):
    rng = np.random.default_rng(seed)
    n_shell = int(round(0.6 * n))
    n_cube = n - n_shell
    v = rng.standard_normal((n_shell, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    theta = np.arccos(np.clip(v[:, 2], -1.0, 1.0))
    phi = np.arctan2(v[:, 1], v[:, 0])
    rad = 1.0 + 0.05 * np.sin(5.0 * theta) * np.cos(3.0 * phi)
    shell = v * rad[:, None]
    cube = rng.uniform(-1.05, 1.05, size=(n_cube, 3))
    pts = np.concatenate([shell, cube])
    return pts[rng.permutation(n)]


def make(name: str, scale: float = 1.0):
    """Returns a dict with src, tgt, values (N x F), basis, nodes_per_cluster."""
    if name == "uniform_20k":
        n = max(int(20_000 * scale), 64)
        src, tgt = _uniform(n, 1), _uniform(n, 2)
        return dict(name=name, src=src, tgt=tgt, values=franke_3d(src)[:, None],
                    basis=WENDLANDC2, nodes_per_cluster=30)
    if name == "grid_blobs_1m":
        n = max(int(1_000_000 * scale), 64)
        if scale == 1.0:
            src, tgt = _grid_blobs(n, 11), _uniform(n, 12)
        else:
            src = _grid_blobs_scaled(n, scale, 11)
            side = max(int(round(100 * scale ** (1.0 / 3.0))), 2) / 100.0
            tgt = _uniform(n, 12, 0.0, side)
        return dict(name=name, src=src, tgt=tgt, values=franke_3d(src)[:, None],
                    basis=WENDLANDC4, nodes_per_cluster=50)
    if name == "shell_4m":
        ns = max(int(4_000_000 * scale), 64)
        nt = max(int(2_000_000 * scale), 64)
        src, tgt = _shell_cube(ns, 21), _shell_cube(nt, 22)
        vals = np.concatenate([franke_3d(src)[:, None], fourier_fields(src, 7, 23)], axis=1)
        return dict(name=name, src=src, tgt=tgt, values=vals, basis=WENDLANDC4,
                    nodes_per_cluster=50)
    if name == "uniform_500k":
        n = max(int(500_000 * scale), 64)
        src, tgt = _uniform(n, 31), _uniform(n, 32)
        vals = np.concatenate([franke_3d(src)[:, None], fourier_fields(src, 3, 33)], axis=1)
        return dict(name=name, src=src, tgt=tgt, values=vals, basis=WENDLANDC4,
                    nodes_per_cluster=50)
    raise KeyError(name)


def _grid_blobs_scaled(n, scale, seed):
    """grid_blobs_1m at n points: the jittered grid keeps its 0.01 spacing
    inside a sub-box of volume `scale`, and the blobs keep sigma 0.02 with
    64 * scale (at least 1) blob centres inside that sub-box, so patch sizes
    and conditioning stay those of the full workload."""
    rng = np.random.default_rng(seed)
    side = scale ** (1.0 / 3.0)
    g = max(int(round(100 * side)), 2)
    n_grid = min(n // 2, g ** 3)
    n_blob = n - n_grid
    cells = rng.choice(g ** 3, size=n_grid, replace=False)
    ijk = np.stack(np.unravel_index(cells, (g, g, g)), axis=1).astype(np.float64)
    grid = (ijk + 0.5) / 100.0 + rng.uniform(-0.3, 0.3, size=(n_grid, 3)) / 100.0
    nb = max(int(round(64 * scale)), 1)
    centres = rng.uniform(0.0, g / 100.0, size=(nb, 3))
    which = rng.integers(0, nb, size=n_blob)
    blobs = centres[which] + rng.normal(0.0, 0.02, size=(n_blob, 3))
    pts = np.concatenate([grid, blobs])
    return pts[rng.permutation(n)]


def many_problems(count: int = 256, seed: int = 41, scale: float = 1.0):
    """The many-uneven-transfers workload: count independent problems with
    source counts log-uniform in [1000, 50000] (times scale), matched target
    counts, points uniform in boxes of side U(0.5, 2), bases uniform over
    C0..C8 and 1-4 Franke/Fourier fields."""
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(50000))) * scale)
        n = max(n, 64)
        side = rng.uniform(0.5, 2.0)
        src = rng.uniform(0.0, side, size=(n, 3))
        tgt = rng.uniform(0.0, side, size=(n, 3))
        basis = int(rng.choice([WENDLANDC0, WENDLANDC2, WENDLANDC4, WENDLANDC6, WENDLANDC8]))
        nf = int(rng.integers(1, 5))
        vals = franke_3d(src / side)[:, None]
        if nf > 1:
            vals = np.concatenate([vals, fourier_fields(src / side, nf - 1, seed * 1000 + i)], axis=1)
        probs.append(dict(src=src, tgt=tgt, values=vals, basis=basis, nodes_per_cluster=50))
    return probs
