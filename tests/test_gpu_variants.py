"""The large-patch engine under each launch parameter the tuner may choose.

The per-GPU tuning file and the environment select, per call, the first tile
column whose update runs on the int8 tensor cores (the columns before it use
the FP64 step kernel), the number of slot groups (streams) and the ring depth
of the backward sweep; PACMAN_B200_INT8=0 keeps every column update in FP64.
Whatever the choice, the transfer is the same to the mixed bound: here each
variant on grid_blobs at scale 0.05 (patches of up to ~3,000 sources, so
every step kernel, the diagonal-tile launches and both sweep rings run)
against the FP64 (reference LU) transfer, with no patch handed to the FP64
fallback."""
import pytest

import pacman_b200 as pacman
from pacman_b200 import workloads as W
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    w = W.make("grid_blobs_1m", scale=0.05)
    v = w["values"][:, 0]
    ref = pacman.rbf.interpolate(3, pacman.execspaces.CUDA, w["basis"], w["src"], v, w["tgt"],
                                 nodes_per_cluster=w["nodes_per_cluster"], precision="fp64")
    return w, v, ref


@pytest.mark.parametrize("env", [
    {"PACMAN_B200_INT8_FROM": "0"},
    {"PACMAN_B200_INT8_FROM": "3"},
    {"PACMAN_B200_INT8_FROM": "6"},
    {"PACMAN_B200_INT8": "0"},
    {"PACMAN_B200_GROUPS": "1"},
    {"PACMAN_B200_GROUPS": "8"},
    {"PACMAN_B200_BACK_STAGES": "6"},
], ids=lambda e: ",".join(f"{k[12:]}={v}" for k, v in e.items()))
def test_launch_variants_give_the_same_transfer(case, env, monkeypatch):
    w, v, ref = case
    for k, val in env.items():
        monkeypatch.setenv(k, val)
    st = {}
    out = pacman.rbf.interpolate(3, pacman.execspaces.CUDA, w["basis"], w["src"], v, w["tgt"],
                                 nodes_per_cluster=w["nodes_per_cluster"], precision="mixed",
                                 stats=st)
    assert st["max_n"] > 2000
    assert st["patches_fallback"] == 0
    assert rel_l2(out, ref) <= 1e-10
