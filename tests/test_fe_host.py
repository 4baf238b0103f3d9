"""NEAREST_NEAREST finite-element transfer on the CPU: the oracle pinned by
the reference's own known answer (tests/test_fe.py:79-95: on the non-"aste"
meshes the targets are the source nodes, and the transfer must return the
source values), its tie rule, and the argument checks of the C ABI and of
pacman_b200.fe.interpolate, which run before any device work."""
import ctypes

import numpy as np
import pytest

import oracle
import pacman_b200 as pacman
from pacman_b200 import _lib


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_oracle_nodes_reproduce_source_values(dim):
    rng = np.random.default_rng(dim)
    S = rng.random((700, dim))
    v = rng.standard_normal(700)
    out, idx = oracle.fe_nearest(dim, S, v, S)
    assert np.array_equal(idx, np.arange(700))
    assert np.array_equal(out, v)


def test_oracle_ties_and_empty():
    S = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 0.0], [1.0, 0.0]])
    v = np.array([1.0, 2.0, 3.0, 4.0])
    T = np.array([[0.5, 0.0], [0.2, 0.0], [0.9, 0.0]])
    out, idx = oracle.fe_nearest(2, S, v, T)
    assert list(idx) == [0, 0, 1]  # equidistant: lowest index
    out, idx = oracle.fe_nearest(2, np.zeros((0, 2)), np.zeros(0), T)
    assert np.all(out == 0.0) and np.all(idx == -1)


def test_abi_rejects_before_device_work():
    lib = _lib.load()
    pts = np.zeros((4, 3))
    vals = np.zeros(4)
    out = np.zeros(4)
    st = np.zeros(4, dtype=np.int32)
    args = lambda dim, method: (dim, method, pts.ctypes.data, 4, vals.ctypes.data, pts.ctypes.data,
                                4, out.ctypes.data, st.ctypes.data, None)
    assert lib.pacman_b200_fe_interpolate(*args(4, 0xF0)) == _lib.ERR_DIMENSION
    assert lib.pacman_b200_fe_interpolate(*args(3, 0xF1)) == _lib.ERR_INVALID
    assert "NEAREST_NEAREST" in _lib.last_error()
    assert lib.pacman_b200_fe_interpolate(3, 0xF0, None, 4, vals.ctypes.data, pts.ctypes.data, 4,
                                          out.ctypes.data, None, None) == _lib.ERR_INVALID
    assert lib.pacman_b200_fe_interpolate(3, 0xF0, pts.ctypes.data, 4, None, pts.ctypes.data, 4,
                                          out.ctypes.data, None, None) == _lib.ERR_INVALID


def test_python_shape_checks():
    S = np.zeros((10, 3))
    fe = pacman.fe
    with pytest.raises(ValueError):
        fe.interpolate(3, 3, fe.methods.NEAREST_NEAREST, S[:, 0], S[:, 0], None, None, None, S)
    with pytest.raises(ValueError):
        fe.interpolate(3, 3, fe.methods.NEAREST_NEAREST, S, S[:5, 0], None, None, None, S)
    with pytest.raises(ValueError):
        fe.interpolate(3, 3, fe.methods.NEAREST_NEAREST, S, S[:, 0], None, None, None, S[:, :2])
    with pytest.raises(RuntimeError):
        fe.interpolate(4, 3, fe.methods.NEAREST_NEAREST, S, S[:, 0], None, None, None, S)
    out, status = fe.interpolate(3, 3, fe.methods.NEAREST_NEAREST, S, S[:, 0], None, None, None,
                                 np.zeros((0, 3)))
    assert out.shape == (0,) and status.shape == (0,)
