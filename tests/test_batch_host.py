"""Host-side checks of the batched entry point: argument validation happens
before any device work, so these run without a GPU."""
import ctypes

import numpy as np
import pytest

from pacman_b200 import _lib
import pacman_b200 as pacman


def _problem(dim=3, fn=0x11, n=10, F=1, m=10):
    pts = np.zeros((max(n, m), 3))
    vals = np.zeros((max(n, 1), F))
    out = np.zeros((max(m, 1), F))
    keep = (pts, vals, out)
    return _lib.Problem(dim, fn, pts.ctypes.data, n, vals.ctypes.data, F, pts.ctypes.data, m,
                        out.ctypes.data), keep


def test_batch_rejects_bad_problem_before_device_work():
    lib = _lib.load()
    cases = [
        (dict(dim=4), _lib.ERR_DIMENSION, "problem 1"),
        (dict(fn=0x77), _lib.ERR_INVALID, "problem 1"),
        (dict(F=9), _lib.ERR_INVALID, "n_fields"),
        (dict(n=-1), _lib.ERR_INVALID, "negative"),
    ]
    for kw, code, text in cases:
        good, k0 = _problem()
        bad, k1 = _problem(**kw)
        arr = (_lib.Problem * 2)(good, bad)
        rc = lib.pacman_b200_rbf_interpolate_batch(arr, 2, None, None)
        assert rc == code, kw
        assert text in _lib.last_error(), (kw, _lib.last_error())


def test_batch_null_arrays_and_counts():
    lib = _lib.load()
    assert lib.pacman_b200_rbf_interpolate_batch(None, 0, None, None) == _lib.OK
    assert lib.pacman_b200_rbf_interpolate_batch(None, 3, None, None) == _lib.ERR_INVALID
    assert lib.pacman_b200_rbf_interpolate_batch(None, -1, None, None) == _lib.ERR_INVALID
    p = _lib.Problem(3, 0x11, None, 5, None, 1, None, 0, None)
    arr = (_lib.Problem * 1)(p)
    assert lib.pacman_b200_rbf_interpolate_batch(arr, 1, None, None) == _lib.ERR_INVALID
    o = _lib.default_options()
    o.relative_overlap = 1.5
    assert lib.pacman_b200_rbf_interpolate_batch(arr, 1, ctypes.byref(o), None) == _lib.ERR_INVALID


def test_python_batch_validation():
    S = np.zeros((10, 3))
    assert pacman.rbf.interpolate_batch([]) == []
    with pytest.raises(ValueError):
        pacman.rbf.interpolate_batch([(3, 0x11, S, S[:, 0])])
    with pytest.raises(ValueError):
        pacman.rbf.interpolate_batch([(3, 0x99, S, S[:, 0], S)])
    with pytest.raises(ValueError):
        pacman.rbf.interpolate_batch([(3, 0x11, S, S[:5, 0], S)])
