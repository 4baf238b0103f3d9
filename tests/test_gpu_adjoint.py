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
