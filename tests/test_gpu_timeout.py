"""A tensor-core pipeline wait that gives up: its patch is marked and solved
again by the FP64 LU path (the reference's algorithm), and the transfer
still meets its bound against the oracle.

The int8 column updates of the mixed Cholesky wait on mbarriers for their
bulk copies and MMAs, each wait bounded; PACMAN_B200_WAIT_LIMIT shortens the
bound to one poll, so the waits give up although nothing is wrong.  The
kernel then drains the copies and MMAs it had issued (with its own, longer
bound), marks the patch (status bit 8) and finishes; the host re-solves the
marked patches by the LU path (bit 16).  No GPU fault is involved: the
copies complete normally, the waits just stop looking early."""
import numpy as np
import pytest

import oracle
import pacman_b200 as pacman
from pacman_b200 import workloads as W
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def test_pipeline_timeout_resolves_patches_by_fp64_lu(monkeypatch):
    # The int8 steps from tile column 0 (the tuned B200 setting), so every
    # patch of the tiled engine (n > 64) reaches a bounded pipeline wait.
    monkeypatch.setenv("PACMAN_B200_INT8_FROM", "0")
    w = W.make("grid_blobs_1m", scale=0.01)  # 21 patches with n > 320, largest 1,692
    S, T, v = w["src"], w["tgt"], w["values"][:, 0]
    ref = oracle.interpolate(3, 0x12, S, v, T, 50)
    plan = pacman.rbf.Plan(3, S, T, precision="mixed")
    out0 = plan.execute(0x12, v)
    assert not (plan.patch_status() & (8 | 16)).any()
    assert rel_l2(out0, ref) <= 1e-10

    monkeypatch.setenv("PACMAN_B200_WAIT_LIMIT", "1")
    st = {}
    out1 = plan.execute(0x12, v, stats=st)
    status = plan.patch_status()
    monkeypatch.delenv("PACMAN_B200_WAIT_LIMIT")
    off, _ = plan.patch_lists("source")
    n = np.diff(off)
    timed = (status & 8) != 0
    assert timed.sum() > 0 and (n[timed] > 64).all()
    assert ((status[timed] & 16) != 0).all()
    assert st["patches_fallback"] >= int(timed.sum())
    assert rel_l2(out1, ref) <= 1e-10
    # The re-solved patches hold the FP64 LU's local values.
    lu = pacman.rbf.Plan(3, S, T, precision="fp64")
    lu.execute(0x12, v)
    toff, _ = plan.patch_lists("target")
    rows = np.concatenate([np.arange(toff[k], toff[k + 1]) for k in np.where(timed)[0]])
    assert rel_l2(plan.local_values()[rows], lu.local_values()[rows]) <= 1e-14

    # Back to the normal bound: no time-outs, the int8 path again.
    out2 = plan.execute(0x12, v)
    assert not (plan.patch_status() & (8 | 16)).any()
    assert np.array_equal(out2, out0)
