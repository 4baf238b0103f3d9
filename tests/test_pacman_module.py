"""``import pacman`` gives the reference's Python module names over the B200
engine (src/pybindings/bindings.cpp:17-93).

The GPU case is the reference's functional test tests/test_rbf-pum.py written
the way that script calls the module (``pacman.rbf.interpolate(3, execspace,
method, sp, sp_values, tp)``, line 58), over its three mesh pairs, five bases
and the execution spaces it lists, with its tolerance: every mesh file name
holds a '3', so rel-L2 < 1.5e-2 against the analytic Franke field
(test_rbf-pum.py:62-74)."""
import numpy as np
import pytest

import pacman
import pacman_b200
from pacman_b200 import workloads as W
from tests.conftest import rel_l2, slab_meshes


def test_module_names_match_the_reference():
    assert pacman.rbf is pacman_b200.rbf and pacman.execspaces is pacman_b200.execspaces
    f = pacman.rbf.functions
    assert [f.WENDLANDC0, f.WENDLANDC2, f.WENDLANDC4, f.WENDLANDC6, f.WENDLANDC8] == \
        [0x10, 0x11, 0x12, 0x13, 0x14]
    e = pacman.execspaces
    assert [e.SERIAL, e.OPENMP, e.THREADS, e.CUDA, e.HIP, e.SYCL] == [0, 1, 2, 3, 4, 5]
    assert callable(pacman.rbf.interpolate) and callable(pacman.fe.interpolate)
    pacman.initialize()
    pacman.finalize()


def test_reference_shape_errors():
    with pytest.raises(ValueError):
        pacman.rbf.interpolate(3, pacman.execspaces.CUDA, pacman.rbf.functions.WENDLANDC2,
                               np.zeros(5), np.zeros(5), np.zeros((4, 3)))


@pytest.mark.gpu
@pytest.mark.parametrize("execspace", ["SERIAL", "OPENMP", "CUDA"])
@pytest.mark.parametrize("method", ["WENDLANDC0", "WENDLANDC2", "WENDLANDC4", "WENDLANDC6",
                                    "WENDLANDC8"])
def test_reference_functional_script(execspace, method):
    meshes = slab_meshes()
    pacman.initialize()
    for src_name, tgt_name in (("0.03", "0.003"), ("0.003", "0.03"), ("0.03", "0.03")):
        sp = meshes[src_name][:, :3].astype(np.float64)
        tp = meshes[tgt_name][:, :3].astype(np.float64)
        sp_values = W.franke_3d(sp)
        tp_values = pacman.rbf.interpolate(3, getattr(pacman.execspaces, execspace),
                                           getattr(pacman.rbf.functions, method), sp, sp_values,
                                           tp)
        assert tp_values.dtype == np.float64 and tp_values.shape == (len(tp),)
        assert rel_l2(tp_values, W.franke_3d(tp)) < 1.5e-2
