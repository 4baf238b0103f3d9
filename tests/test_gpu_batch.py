"""Batched transfers (pacman_b200_rbf_interpolate_batch) through the C ABI.

Each problem of a batch must give what a single-problem call gives for it
(the merged solve runs the same per-patch arithmetic), and so match the CPU
oracle within the transfer's tolerances: rel-L2 1e-12 in FP64, 1e-10 mixed."""
import numpy as np
import pytest

import oracle
import pacman_b200 as pacman
from pacman_b200 import workloads as W
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-10
TOL_SAME = 1e-13  # batch against single calls of the same engine
CUDA = pacman.execspaces.CUDA


def _problems(count, scale, seed=41):
    probs = W.many_problems(count=count, seed=seed, scale=scale)
    return [(3, q["basis"], q["src"], q["values"] if q["values"].shape[1] > 1
             else q["values"][:, 0], q["tgt"]) for q in probs]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_calls(precision):
    probs = _problems(24, 0.1)
    st = {}
    outs = pacman.rbf.interpolate_batch(probs, precision=precision, stats=st)
    assert len(outs) == len(probs)
    total_patches = 0
    for (dim, basis, S, v, T), out in zip(probs, outs):
        one = {}
        ref = pacman.rbf.interpolate(dim, CUDA, basis, S, v, T, precision=precision, stats=one)
        assert out.shape == ref.shape
        assert rel_l2(out, ref) <= TOL_SAME
        total_patches += one["num_patches"]
    assert st["num_patches"] == total_patches


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_FP64), ("mixed", TOL_MIXED)])
def test_batch_matches_oracle(precision, tol):
    probs = _problems(8, 0.05, seed=7)
    outs = pacman.rbf.interpolate_batch(probs, precision=precision)
    for (dim, basis, S, v, T), out in zip(probs, outs):
        ref = oracle.interpolate(dim, basis, S, v, T, 50)
        assert rel_l2(out, ref) <= tol


def test_batch_large_patches():
    # Dense blobs: patches above the small-kernel sizes go through the
    # blocked engine, merged across problems.
    a = W.make("grid_blobs_1m", scale=0.01)
    b = W.make("grid_blobs_1m", scale=0.02)
    probs = [(3, 0x12, a["src"], a["values"][:, :1], a["tgt"]),
             (3, 0x12, b["src"], b["values"][:, 0], b["tgt"])]
    for precision, tol in (("fp64", TOL_FP64), ("mixed", TOL_MIXED)):
        outs = pacman.rbf.interpolate_batch(probs, precision=precision)
        for (dim, basis, S, v, T), out in zip(probs, outs):
            ref = oracle.interpolate(dim, basis, S, np.ravel(v), T, 50)
            assert rel_l2(np.ravel(out), ref) <= tol


def test_batch_mixed_dims_and_edges():
    rng = np.random.default_rng(5)
    S1, T1 = rng.random((900, 1)), rng.random((700, 1))
    S2, T2 = rng.random((2500, 2)), rng.random((2000, 2))
    S3, T3 = rng.random((3000, 3)), rng.random((2500, 3))
    v1 = np.cos(3 * S1[:, 0])
    v2 = np.c_[np.sin(4 * S2[:, 0]) * np.cos(3 * S2[:, 1]), S2[:, 0] * S2[:, 1]]
    v3 = W.franke_3d(S3)
    far = rng.random((40, 3)) + 10.0
    probs = [
        (1, 0x10, S1, v1, T1),
        (3, 0x11, S3, v3, np.concatenate([T3, far])),  # targets outside every patch
        (2, 0x13, S2, v2, T2),
        (3, 0x11, S3, v3, np.zeros((0, 3))),           # no targets
        (3, 0x11, np.zeros((0, 3)), np.zeros(0), T3[:10]),  # no sources: zeros
        (3, 0x14, S3[:20], v3[:20], T3[:30]),          # fewer sources than a cluster
    ]
    outs = pacman.rbf.interpolate_batch(probs)
    assert outs[3].shape == (0,)
    assert np.all(outs[4] == 0.0)
    assert np.all(outs[1][-40:] == 0.0)
    for i in (0, 1, 2, 5):
        dim, basis, S, v, T = probs[i]
        single = pacman.rbf.interpolate(dim, CUDA, basis, S, v, T)
        assert rel_l2(outs[i], single) <= TOL_SAME
        for f in range(1 if v.ndim == 1 else v.shape[1]):
            vf = v if v.ndim == 1 else v[:, f]
            of = outs[i] if v.ndim == 1 else outs[i][:, f]
            assert rel_l2(of, oracle.interpolate(dim, basis, S, vf, T, 50)) <= TOL_FP64


def test_batch_torch_device_tensors():
    torch = pytest.importorskip("torch")
    probs = _problems(6, 0.05, seed=3)
    host = pacman.rbf.interpolate_batch(probs)
    dev = [(d, b, torch.tensor(S, device="cuda"), torch.tensor(v, device="cuda"),
            torch.tensor(T, device="cuda")) for d, b, S, v, T in probs]
    outs = pacman.rbf.interpolate_batch(dev)
    for h, o in zip(host, outs):
        assert o.is_cuda
        assert rel_l2(o.cpu().numpy(), h) <= TOL_SAME


def test_batch_reports_failing_problem():
    rng = np.random.default_rng(1)
    S = rng.random((500, 3))
    good = (3, 0x11, S, W.franke_3d(S), S[:100])
    bad = (3, 0x11, S, W.franke_3d(S), rng.random((100, 2)))
    with pytest.raises(ValueError):
        pacman.rbf.interpolate_batch([good, bad])
