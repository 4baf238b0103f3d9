"""Moving least squares on the GPU (pacman_b200_mls_interpolate, k_mls)
against the CPU oracle, bit for bit: the neighbour search, the weights, the
moment matrix and the Jacobi pseudo-inverse run the same IEEE operations in
the same order on both sides (no contraction in either).  Also the
reference's MLS known answers (tests/test_mls.py:83-92,
tests/test_cpp_mls_interface.cpp:148-151) through pacman.MLS.interpolate and
through the C++ symbol PACMAN::MLS_interpolate."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import pacman
from pacman_b200 import workloads as W
from tests.conftest import ROOT

pytestmark = pytest.mark.gpu
CUDA = pacman.execspaces.CUDA


def _grid(n, dim):
    axes = np.meshgrid(*([np.linspace(0.0, 1.0, n)] * dim), indexing="ij")
    return np.stack([a.ravel() for a in axes], axis=1)


def _same(dim, S, f, T):
    out = pacman.MLS.interpolate(dim, CUDA, S, f, T)
    ref = oracle.mls_interpolate(dim, S, f, T)
    assert np.array_equal(out, ref), np.abs(out - ref).max()
    return out


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_reference_grid_known_answer(dim):
    g = _grid(20, dim)
    v = W.franke(g)
    out = _same(dim, g, v, g)
    assert np.linalg.norm(out - v) / np.linalg.norm(v) < 1e-4


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_random_clouds(dim):
    rng = np.random.default_rng(30 + dim)
    S = rng.random((6000, dim))
    T = rng.random((4000, dim))
    _same(dim, S, W.franke(S), T)


def test_clustered_sources_and_far_targets():
    rng = np.random.default_rng(41)
    centres = rng.random((8, 3))
    S = centres[rng.integers(0, 8, 20000)] + rng.normal(0.0, 0.02, size=(20000, 3))
    T = np.concatenate([rng.random((3000, 3)), rng.random((200, 3)) * 4.0 + 2.0])
    _same(3, S, np.sin(3 * S[:, 0]) + S[:, 1] * S[:, 2], T)


def test_duplicate_sources_and_planar_clouds():
    rng = np.random.default_rng(42)
    base = rng.random((1500, 3))
    S = np.concatenate([base, base[:700]])          # exact distance ties
    f = rng.standard_normal(len(S))
    _same(3, S, f, rng.random((1500, 3)))
    P = np.c_[rng.random((3000, 2)), np.zeros(3000)]  # sources on the plane z = 0
    T = np.c_[rng.random((1000, 2)), rng.choice([0.0, 0.05], size=1000)]
    _same(3, P, W.franke(P), T)


@pytest.mark.parametrize("dim,n", [(3, 1), (3, 4), (2, 2), (1, 2)])
def test_fewer_sources_than_the_basis(dim, n):
    rng = np.random.default_rng(43)
    S = rng.random((n, dim))
    _same(dim, S, rng.random(n), rng.random((500, dim)))


def test_no_sources_and_no_targets():
    T = np.random.default_rng(44).random((100, 3))
    out = pacman.MLS.interpolate(3, CUDA, np.zeros((0, 3)), np.zeros(0), T)
    assert out.shape == (100,) and (out == 0).all()
    out = pacman.MLS.interpolate(3, CUDA, T, np.ones(100), np.zeros((0, 3)))
    assert out.shape == (0,)


def test_torch_device_inputs_match_host_inputs():
    import torch
    rng = np.random.default_rng(45)
    S = rng.random((5000, 3))
    T = rng.random((3000, 3))
    f = W.franke(S)
    host = pacman.MLS.interpolate(3, CUDA, S, f, T)
    dev = pacman.MLS.interpolate(3, CUDA, torch.from_numpy(S).cuda(), torch.from_numpy(f).cuda(),
                                 torch.from_numpy(T).cuda())
    assert dev.is_cuda
    assert np.array_equal(dev.cpu().numpy(), host)


def test_million_points_sampled_against_the_oracle():
    """1M uniform sources -> 1M uniform targets in 3D; the oracle recomputes
    2,000 sampled targets, which must match exactly.
    The fit's own error against Franke's function is ~7e-3 rel-L2 here (ten
    neighbours for ten basis functions interpolate, and some random
    neighbour sets are close to singular), so the last check is a loose
    sanity bound."""
    rng = np.random.default_rng(46)
    S = rng.random((1_000_000, 3))
    T = rng.random((1_000_000, 3))
    f = W.franke(S)
    out = pacman.MLS.interpolate(3, CUDA, S, f, T)
    pick = rng.choice(len(T), size=2000, replace=False)
    ref = oracle.mls_interpolate(3, S, f, T[pick])
    assert np.array_equal(out[pick], ref)
    assert np.linalg.norm(out - W.franke(T)) / np.linalg.norm(W.franke(T)) < 2e-2


CPP_MLS = r"""
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <vector>
#include "pacman_rbf.hpp"

static double franke3(double x, double y, double z) {
  return 0.75 * std::exp(-((9 * x - 2) * (9 * x - 2) + (9 * y - 2) * (9 * y - 2) +
                           (9 * z - 2) * (9 * z - 2)) / 4.0) +
         0.75 * std::exp(-((9 * x + 1) * (9 * x + 1) / 49.0 + (9 * y + 1) / 10.0 +
                           (9 * z + 1) / 10.0)) +
         0.5 * std::exp(-((9 * x - 7) * (9 * x - 7) + (9 * y - 3) * (9 * y - 3) +
                          (9 * z - 5) * (9 * z - 5)) / 4.0) -
         0.2 * std::exp(-((9 * x - 4) * (9 * x - 4) + (9 * y - 7) * (9 * y - 7) +
                          (9 * z - 5) * (9 * z - 5)));
}

int main() {
  const int N = 20;
  std::vector<double> p, v;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < N; ++k) {
        const double x = i / double(N - 1), y = j / double(N - 1), z = k / double(N - 1);
        p.insert(p.end(), {x, y, z});
        v.push_back(franke3(x, y, z));
      }
  const int n = N * N * N;
  PACMAN::MLSInterpolateResult r =
      PACMAN::MLS_interpolate(3, PACMAN::ExecSpaces::CUDA, p.data(), n, v.data(), p.data(), n);
  double num = 0, den = 0;
  for (int i = 0; i < n; ++i) {
    num += (r.targetValues[i] - v[i]) * (r.targetValues[i] - v[i]);
    den += v[i] * v[i];
  }
  const double err = std::sqrt(num / den);
  std::printf("rel_l2 %.3e\n", err);
  bool threw = false;
  try {
    PACMAN::MLS_interpolate(3, PACMAN::ExecSpaces::CUDA, nullptr, n, v.data(), p.data(), n);
  } catch (const std::invalid_argument &) {
    threw = true;
  }
  return (err < 1e-4 && threw) ? 0 : 1;
}
"""


def test_cpp_mls_dropin(tmp_path):
    """tests/test_cpp_mls_interface.cpp's case ("same": the 20^3 grid onto
    itself, rel-L2 < 1e-4) through PACMAN::MLS_interpolate."""
    src = tmp_path / "t.cpp"
    src.write_text(CPP_MLS)
    exe = tmp_path / "t"
    libdir = os.path.join(ROOT, "pacman_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", str(src), "-I", os.path.join(ROOT, "include"),
                    "-L", libdir, "-lpacman_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
