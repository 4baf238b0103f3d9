"""The C-ABI library loads and exports every declared symbol; the host-side
argument checks mirror the reference's.  No GPU needed."""
import ctypes
import os
import re

import numpy as np
import pytest

import pacman_b200 as pacman
from pacman_b200 import _lib
from tests.conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pacman_b200.h")).read()
    return sorted(set(re.findall(r"PACMAN_B200_API\s+[\w\s\*]*?\b(pacman_b200_\w+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES)
    assert _lib.load().pacman_b200_abi_version() == 6


def test_cpp_dropin_symbol_exported():
    out = os.popen(f"nm -D --defined-only {_lib.LIB_PATH}").read()
    assert "_ZN6PACMAN15rbf_interpolateEihhPdiS0_S0_i" in out


def test_default_options_are_the_reference_defaults():
    o = _lib.default_options()
    assert (o.nodes_per_cluster, o.relative_overlap, o.support_radius) == (50, 0.15, 0.1)
    assert o.precision == _lib.FP64 and o.device == -1 and not o.stream


def test_constants_match_reference():
    f = pacman.rbf.functions
    assert (f.WENDLANDC0, f.WENDLANDC2, f.WENDLANDC4, f.WENDLANDC6, f.WENDLANDC8) == (
        0x10, 0x11, 0x12, 0x13, 0x14)
    e = pacman.execspaces
    assert (e.SERIAL, e.OPENMP, e.THREADS, e.CUDA, e.HIP, e.SYCL) == (0, 1, 2, 3, 4, 5)
    assert "CUDA" in e.available()


@pytest.mark.parametrize("sp,sv,tp,exc", [
    (np.zeros(5), np.zeros(5), np.zeros((4, 3)), ValueError),          # source not 2-d
    (np.zeros((5, 3)), np.zeros(5), np.zeros(4), ValueError),          # target not 2-d
    (np.zeros((5, 3)), np.zeros(5), np.zeros((4, 2)), ValueError),     # dims mismatch
    (np.zeros((5, 3)), np.zeros(6), np.zeros((4, 3)), ValueError),     # values count
])
def test_shape_checks(sp, sv, tp, exc):
    with pytest.raises(exc):
        pacman.rbf.interpolate(3, pacman.execspaces.CUDA, pacman.rbf.functions.WENDLANDC2,
                               sp, sv, tp)


def test_bad_dimension_and_selectors():
    z = np.zeros((5, 4))
    with pytest.raises(RuntimeError):
        pacman.rbf.interpolate(4, 3, 0x11, z, np.zeros(5), z)
    with pytest.raises(ValueError):
        pacman.rbf.interpolate(3, 3, 0x20, np.zeros((5, 3)), np.zeros(5), np.zeros((4, 3)))
    with pytest.raises(ValueError):
        pacman.rbf.interpolate(3, 9, 0x11, np.zeros((5, 3)), np.zeros(5), np.zeros((4, 3)))


def test_c_abi_validates_before_touching_the_device():
    lib = _lib.load()
    out = np.zeros(4)
    p = np.zeros((4, 3))
    v = np.zeros(4)
    rc = lib.pacman_b200_rbf_interpolate(4, 0x11, p.ctypes.data, 4, v.ctypes.data, 1,
                                         p.ctypes.data, 4, out.ctypes.data, None, None)
    assert rc == _lib.ERR_DIMENSION
    rc = lib.pacman_b200_rbf_interpolate(3, 0x42, p.ctypes.data, 4, v.ctypes.data, 1,
                                         p.ctypes.data, 4, out.ctypes.data, None, None)
    assert rc == _lib.ERR_INVALID and "selector" in _lib.last_error()
    rc = lib.pacman_b200_rbf_interpolate(3, 0x11, None, 4, v.ctypes.data, 1, p.ctypes.data, 4,
                                         out.ctypes.data, None, None)
    assert rc == _lib.ERR_INVALID and "sourcePoints is null" in _lib.last_error()
    rc = lib.pacman_b200_rbf_interpolate(3, 0x11, p.ctypes.data, 4, None, 1, p.ctypes.data, 4,
                                         out.ctypes.data, None, None)
    assert rc == _lib.ERR_INVALID and "sourceValues is null" in _lib.last_error()
    rc = lib.pacman_b200_rbf_interpolate(3, 0x11, p.ctypes.data, 4, v.ctypes.data, 9,
                                         p.ctypes.data, 4, out.ctypes.data, None, None)
    assert rc == _lib.ERR_INVALID
    o = _lib.default_options()
    o.relative_overlap = 1.5
    rc = lib.pacman_b200_rbf_interpolate(3, 0x11, p.ctypes.data, 4, v.ctypes.data, 1,
                                         p.ctypes.data, 4, out.ctypes.data, ctypes.byref(o), None)
    assert rc == _lib.ERR_INVALID and "overlap" in _lib.last_error()


def test_header_and_python_signatures_agree():
    src = open(os.path.join(ROOT, "include", "pacman_b200.h")).read()
    for name, (res, args) in _lib.SIGNATURES.items():
        m = re.search(r"PACMAN_B200_API\s+[\w\s\*]*?\b" + name + r"\s*\(([^)]*)\)", src, re.S)
        assert m, name
        params = [p for p in m.group(1).split(",") if p.strip() and p.strip() != "void"]
        assert len(params) == len(args), name
