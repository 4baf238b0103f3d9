"""Adjoint of the transfer (no reference counterpart): the transpose with
respect to the source values against the explicitly assembled FP64 operator,
the gradient with respect to the target coordinates against central finite
differences (h = 1e-6), and the torch.autograd.Function."""
import numpy as np
import pytest

import oracle
import pacman_b200 as pacman
from pacman_b200 import workloads as W
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(n=1500, m=1200, seed=5):
    rng = np.random.default_rng(seed)
    S, T = rng.random((n, 3)), rng.random((m, 3)) * 0.9 + 0.05
    return S, T


def _dense_operator(plan, n, basis):
    """M[:, i] = transfer of the i-th unit vector (8 columns per call)."""
    cols = []
    for i0 in range(0, n, 8):
        E = np.zeros((n, 8))
        for j in range(min(8, n - i0)):
            E[i0 + j, j] = 1.0
        cols.append(plan.execute(basis, E)[:, : min(8, n - i0)])
    return np.concatenate(cols, axis=1)


@pytest.mark.parametrize("big_n", [None, "8"])
def test_values_adjoint_is_the_operator_transpose(big_n, monkeypatch):
    if big_n:
        monkeypatch.setenv("PACMAN_B200_BIG_N", big_n)  # route patches through the blocked engine
    S, T = _case()
    basis = 0x12
    plan = pacman.rbf.Plan(3, S, T, nodes_per_cluster=30)
    M = _dense_operator(plan, S.shape[0], basis)
    G = np.random.default_rng(9).standard_normal((T.shape[0], 3))
    plan.execute(basis, np.random.default_rng(2).standard_normal((S.shape[0], 3)),
                 save_for_adjoint=True)
    gv, _ = plan.adjoint(G, values=True, targets=False)
    assert rel_l2(gv, M.T @ G) <= 1e-11


def test_values_adjoint_against_oracle_operator():
    # Explicit FP64 operator from the CPU oracle (unit vectors, 8 per solve).
    S, T = _case(700, 600, seed=6)
    basis = 0x11
    ref = oracle.build(3, S, T, 30)
    cols = []
    for i0 in range(0, S.shape[0], 8):
        E = np.zeros((S.shape[0], 8))
        w = min(8, S.shape[0] - i0)
        for j in range(w):
            E[i0 + j, j] = 1.0
        cols.append(ref.solve(basis, E)[0][:, :w])
    M = np.concatenate(cols, axis=1)
    G = np.random.default_rng(4).standard_normal(T.shape[0])
    plan = pacman.rbf.Plan(3, S, T, nodes_per_cluster=30)
    plan.execute(basis, np.ones(S.shape[0]), save_for_adjoint=True)
    gv, _ = plan.adjoint(G, values=True, targets=False)
    assert rel_l2(gv, M.T @ G) <= 1e-11


def _objective(S, T, V, G, basis, npc):
    plan = pacman.rbf.Plan(3, S, T, nodes_per_cluster=npc)
    out = plan.execute(basis, V)
    return float(np.sum(out * G)), plan


@pytest.mark.parametrize("basis,big_n", [(0x11, None), (0x12, None), (0x13, None), (0x12, "8")])
def test_target_gradient_central_differences(basis, big_n, monkeypatch):
    if big_n:
        monkeypatch.setenv("PACMAN_B200_BIG_N", big_n)
    # Uniform 500k -> 500k workload shape at 2k points, 4 fields, h = 1e-6,
    # 64 random unit directions over all target coordinates.
    w = W.make("uniform_500k", scale=0.004)
    S, T, V = w["src"], w["tgt"], w["values"]
    G = np.random.default_rng(11).standard_normal((T.shape[0], V.shape[1]))
    plan = pacman.rbf.Plan(3, S, T)
    plan.execute(basis, V, save_for_adjoint=True)
    _, gt = plan.adjoint(G, values=False, targets=True)
    base_lists = [plan.patch_lists("source"), plan.patch_lists("target")]
    rng = np.random.default_rng(12)
    h = 1e-6
    checked = 0
    for _ in range(64):
        D = rng.standard_normal(T.shape)
        D /= np.linalg.norm(D)
        lp, pp = _objective(S, T + h * D, V, G, basis, 50)
        lm, pm = _objective(S, T - h * D, V, G, basis, 50)
        same = all(np.array_equal(a, b) for p2 in (pp, pm)
                   for a, b in zip(base_lists[1], p2.patch_lists("target")))
        if not same:
            continue  # a target crossed a patch boundary: not differentiable there
        fd = (lp - lm) / (2 * h)
        an = float(np.sum(gt * D))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
        checked += 1
    assert checked >= 48


def test_values_gradient_central_differences():
    w = W.make("uniform_500k", scale=0.004)
    S, T, V = w["src"], w["tgt"], w["values"]
    G = np.random.default_rng(13).standard_normal((T.shape[0], V.shape[1]))
    plan = pacman.rbf.Plan(3, S, T)
    plan.execute(0x12, V, save_for_adjoint=True)
    gv, _ = plan.adjoint(G, values=True, targets=False)
    rng = np.random.default_rng(14)
    for _ in range(8):
        D = rng.standard_normal(V.shape)
        fd = (np.sum(plan.execute(0x12, V + 1e-6 * D) * G)
              - np.sum(plan.execute(0x12, V - 1e-6 * D) * G)) / 2e-6
        assert abs(fd - np.sum(gv * D)) <= 1e-7 * max(1.0, abs(fd))


def test_autograd_function_matches_plan_adjoint():
    torch = pytest.importorskip("torch")
    from pacman_b200.autograd import rbf_pum_transfer
    w = W.make("uniform_500k", scale=0.004)
    S = torch.tensor(w["src"], device="cuda")
    T = torch.tensor(w["tgt"], device="cuda", requires_grad=True)
    V = torch.tensor(w["values"], device="cuda", requires_grad=True)
    G = torch.randn(T.shape[0], V.shape[1], dtype=torch.float64, device="cuda")
    out = rbf_pum_transfer(S, V, T, 0x12)
    (out * G).sum().backward()
    plan = pacman.rbf.Plan(3, w["src"], w["tgt"])
    plan.execute(0x12, w["values"], save_for_adjoint=True)
    gv, gt = plan.adjoint(G.cpu().numpy())
    assert out.is_cuda and V.grad.is_cuda and T.grad.is_cuda
    assert rel_l2(V.grad.cpu().numpy(), gv) <= 1e-13
    assert rel_l2(T.grad.cpu().numpy(), gt) <= 1e-13


# ---------------------------------------------------------------------------
# Precision "mixed": the forward solves run the int8 tensor-core Cholesky and
# save their coefficients; the adjoint's transpose solves stay FP64.
# ---------------------------------------------------------------------------

def _blobs_10k():
    # Patches of up to ~1,700 sources: the large ones take the int8 steps.
    w = W.make("grid_blobs_1m", scale=0.01)
    return w["src"], w["tgt"], np.stack([w["values"][:, 0], np.sin(3 * w["src"][:, 1])], 1)


def test_mixed_adjoint_agrees_with_fp64():
    S, T, V = _blobs_10k()
    G = np.random.default_rng(21).standard_normal((T.shape[0], V.shape[1]))
    grads = {}
    for precision in ("fp64", "mixed"):
        plan = pacman.rbf.Plan(3, S, T, precision=precision)
        plan.execute(0x12, V, save_for_adjoint=True)
        grads[precision] = plan.adjoint(G)
    assert rel_l2(grads["mixed"][0], grads["fp64"][0]) <= 1e-10
    assert rel_l2(grads["mixed"][1], grads["fp64"][1]) <= 1e-10


def test_mixed_target_gradient_central_differences():
    S, T, V = _blobs_10k()
    G = np.random.default_rng(22).standard_normal((T.shape[0], V.shape[1]))
    plan = pacman.rbf.Plan(3, S, T, precision="mixed")
    plan.execute(0x12, V, save_for_adjoint=True)
    _, gt = plan.adjoint(G, values=False, targets=True)
    base = plan.patch_lists("target")
    rng = np.random.default_rng(23)
    h, checked = 1e-6, 0
    for _ in range(16):
        D = rng.standard_normal(T.shape)
        D /= np.linalg.norm(D)
        obj, same = [], True
        for sgn in (1.0, -1.0):
            pl = pacman.rbf.Plan(3, S, T + sgn * h * D, precision="mixed")
            obj.append(float(np.sum(pl.execute(0x12, V) * G)))
            same &= all(np.array_equal(a, b) for a, b in zip(base, pl.patch_lists("target")))
        if not same:
            continue
        fd = (obj[0] - obj[1]) / (2 * h)
        an = float(np.sum(gt * D))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)
        checked += 1
    assert checked >= 12


# ---------------------------------------------------------------------------
# The adjoint workload at its full size: 500,000 uniform sources -> 500,000
# uniform targets, Wendland C4, 4 fields, upstream gradients N(0, 1).
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uniform_500k_central_differences(precision):
    w = W.make("uniform_500k")
    S, T, V = w["src"], w["tgt"], w["values"]
    G = np.random.default_rng(31).standard_normal((T.shape[0], V.shape[1]))
    plan = pacman.rbf.Plan(3, S, T, precision=precision)
    plan.execute(0x12, V, save_for_adjoint=True)
    gv, gt = plan.adjoint(G)
    base = plan.patch_lists("target")
    rng = np.random.default_rng(32)
    h = 1e-6
    # Values: the transfer is linear in them, so central differences are
    # exact up to rounding, 64 random directions.
    for _ in range(64):
        D = rng.standard_normal(V.shape)
        fd = (np.sum(plan.execute(0x12, V + h * D) * G)
              - np.sum(plan.execute(0x12, V - h * D) * G)) / (2 * h)
        an = float(np.sum(gv * D))
        assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (fd, an)
    # Target coordinates: 64 random unit directions over all 1.5M coordinates
    # (directions whose perturbation moves a target across a patch boundary
    # are skipped: the transfer is not differentiable there).
    # The objective sums 2M products out * G; each output carries rounding of
    # order eps |out|, so two evaluations h apart differ by up to about
    # eps * sum |out * G| beyond the true change: that, over 2h, is the
    # central difference's own error at this size (~1e-4 here), added to the
    # relative bound of the small cases.
    noise = np.finfo(np.float64).eps * float(np.sum(np.abs(plan.execute(0x12, V) * G))) / (2 * h)
    checked = 0
    for _ in range(64):
        D = rng.standard_normal(T.shape)
        D /= np.linalg.norm(D)
        obj, same = [], True
        for sgn in (1.0, -1.0):
            pl = pacman.rbf.Plan(3, S, T + sgn * h * D, precision=precision)
            obj.append(float(np.sum(pl.execute(0x12, V) * G)))
            same &= all(np.array_equal(a, b) for a, b in zip(base, pl.patch_lists("target")))
            pl.close()
        if not same:
            continue
        fd = (obj[0] - obj[1]) / (2 * h)
        an = float(np.sum(gt * D))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)) + noise, (fd, an, noise)
        checked += 1
    assert checked >= 48


def test_uniform_500k_subset_operator_transpose():
    """The explicit FP64 operator of a 5,000-point subset of the adjoint
    workload (its first 5,000 sources and targets), assembled column by
    column from unit vectors, against the adjoint in both precisions."""
    w = W.make("uniform_500k")
    S, T = w["src"][:5000], w["tgt"][:5000]
    plan = pacman.rbf.Plan(3, S, T)
    M = _dense_operator(plan, S.shape[0], 0x12)
    G = np.random.default_rng(33).standard_normal((T.shape[0], 4))
    ref = M.T @ G
    for precision, tol in (("fp64", 1e-11), ("mixed", 1e-10)):
        p = pacman.rbf.Plan(3, S, T, precision=precision)
        p.execute(0x12, w["values"][:5000], save_for_adjoint=True)
        gv, _ = p.adjoint(G, values=True, targets=False)
        assert rel_l2(gv, ref) <= tol, precision
