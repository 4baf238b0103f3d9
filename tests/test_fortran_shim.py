"""The C entry points of the reference's Fortran module
(src/fortran_interface.h:69-151) exported by libpacman_b200.so.

The Fortran module calls pacman_rbf_interpolate_c, pacman_fe_interpolate_c
and pacman_mls_interpolate_c through ISO_C_BINDING and reads their integer
return code: 0, or -1 when the C++ call threw a std::exception, -2 for
anything else (src/fortran_interface.cpp:84-90).  gfortran is not in this image, so these
tests bind the same C signatures through ctypes, which is what the module's
interface blocks do.  The GPU cases repeat the reference's Fortran known-answer
test (tests/test_fortran_rbf_interface.f90: 20^3 grid onto itself, rel-L2 <
1e-8 for all five bases) through the shim."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from pacman_b200 import _lib
from tests.conftest import ROOT, grid_cloud, rel_l2

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _shim():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    lib.pacman_rbf_interpolate_c.restype = ctypes.c_int
    lib.pacman_rbf_interpolate_c.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D,
                                             ctypes.c_int, _D, _D, ctypes.c_int, _D]
    lib.pacman_fe_interpolate_c.restype = ctypes.c_int
    lib.pacman_fe_interpolate_c.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D,
                                            ctypes.c_int, _D, _I, ctypes.c_int, _I, ctypes.c_int,
                                            _I, _D, ctypes.c_int, _D, _I]
    lib.pacman_mls_interpolate_c.restype = ctypes.c_int
    lib.pacman_mls_interpolate_c.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D,
                                             _D, ctypes.c_int, _D]
    lib.pacman_best_execspace_c.restype = ctypes.c_int
    return lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _rbf(lib, dim, fn, sp, sv, tp, out, n=None, m=None):
    return lib.pacman_rbf_interpolate_c(dim, 3, fn, _dp(sp), len(sp) if n is None else n, _dp(sv),
                                        _dp(tp), len(tp) if m is None else m, _dp(out))


def test_shim_symbols_exported_with_c_linkage():
    src = open(os.path.join(ROOT, "include", "pacman_fortran_shim.h")).read()
    names = re.findall(r"PACMAN_SHIM_API\s+[\w\s\*]*?\b(pacman_\w+_c)\s*\(", src)
    assert set(names) == {"pacman_kokkos_initialize_c", "pacman_kokkos_finalize_c",
                          "pacman_best_execspace_c", "pacman_rbf_interpolate_c",
                          "pacman_fe_interpolate_c", "pacman_mls_interpolate_c"}
    out = os.popen(f"nm -D --defined-only {_lib.LIB_PATH}").read()
    for n in names:
        assert re.search(r"\bT " + n + r"$", out, re.M), n  # unmangled: extern "C"


def test_shim_init_finalize_and_best_execspace():
    lib = _shim()
    lib.pacman_kokkos_initialize_c()
    lib.pacman_kokkos_finalize_c()
    assert lib.pacman_best_execspace_c() == 0x03


def test_shim_maps_exceptions_to_minus_one(capfd):
    """Argument errors are std::exceptions in the C++ API and come back as -1
    with the message on stderr, before any device work."""
    lib = _shim()
    p = np.zeros((4, 3))
    v = np.zeros(4)
    out = np.zeros(4)
    assert _rbf(lib, 4, 0x11, p, v, p, out) == -1            # runtime_error: dimension
    assert "dimension" in capfd.readouterr().err
    assert _rbf(lib, 3, 0x42, p, v, p, out) == -1            # invalid_argument: basis
    assert "pacman_rbf_interpolate_c: Unsupported RBF function" in capfd.readouterr().err
    assert lib.pacman_rbf_interpolate_c(3, 3, 0x11, None, 4, _dp(v), _dp(p), 4, _dp(out)) == -1
    assert "sourcePoints is null" in capfd.readouterr().err
    assert lib.pacman_rbf_interpolate_c(3, 9, 0x11, _dp(p), 4, _dp(v), _dp(p), 4, _dp(out)) == -1
    assert lib.pacman_rbf_interpolate_c(3, 3, 0x11, _dp(p), 4, _dp(v), _dp(p), 4, None) == -1
    # No targets: nothing to do, success, buffer untouched.
    assert lib.pacman_rbf_interpolate_c(3, 3, 0x11, _dp(p), 4, _dp(v), _dp(p), 0, None) == 0
    st = np.zeros(4, dtype=np.int32)
    # FE: a mesh-based method is not served by the engine.
    rc = lib.pacman_fe_interpolate_c(3, 3, 0xF1, _dp(p), 4, _dp(v), None, 0, None, 0, None,
                                     _dp(p), 4, _dp(out), st.ctypes.data_as(_I))
    assert rc == -1 and "NEAREST_NEAREST" in capfd.readouterr().err
    # MLS (src/fortran_interface.cpp:138-164): the same -1 mapping.
    assert lib.pacman_mls_interpolate_c(4, 3, _dp(p), 4, _dp(v), _dp(p), 4, _dp(out)) == -1
    assert "pacman_mls_interpolate_c: The dimension" in capfd.readouterr().err
    assert lib.pacman_mls_interpolate_c(3, 3, _dp(p), 4, None, _dp(p), 4, _dp(out)) == -1
    assert "sourceValues is null" in capfd.readouterr().err
    assert lib.pacman_mls_interpolate_c(3, 3, _dp(p), 4, _dp(v), _dp(p), 4, None) == -1
    assert lib.pacman_mls_interpolate_c(3, 3, _dp(p), 4, _dp(v), _dp(p), 0, None) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("fn", [0x10, 0x11, 0x12, 0x13, 0x14])
def test_shim_fortran_known_answer(fn):
    """tests/test_fortran_rbf_interface.f90: the 20^3 grid onto itself
    reproduces the source values to rel-L2 < 1e-8, here through the C shim;
    the values equal the C ABI's FP64 transfer bit for bit."""
    lib = _shim()
    g = grid_cloud(20)
    v = np.sin(3 * g[:, 0]) + g[:, 1] * g[:, 2]
    out = np.full(len(g), np.nan)
    assert _rbf(lib, 3, fn, g, v, g, out) == 0
    assert rel_l2(out, v) < 1e-8
    ref = np.zeros(len(g))
    rc = _lib.load().pacman_b200_rbf_interpolate(3, fn, g.ctypes.data, len(g), v.ctypes.data, 1,
                                                 g.ctypes.data, len(g), ref.ctypes.data, None,
                                                 None)
    assert rc == 0
    assert np.array_equal(out, ref)


@pytest.mark.gpu
def test_shim_rbf_matches_oracle():
    rng = np.random.default_rng(5)
    sp = rng.random((3000, 3))
    tp = rng.random((2500, 3))
    sv = np.cos(4 * sp[:, 0]) * sp[:, 1]
    out = np.zeros(len(tp))
    assert _rbf(_shim(), 3, 0x11, sp, sv, tp, out) == 0
    ref = oracle.interpolate(3, 0x11, sp, sv, tp, 50)
    assert rel_l2(out, ref) < 1e-12


@pytest.mark.gpu
def test_shim_fe_nearest_nearest():
    rng = np.random.default_rng(6)
    sp = rng.random((2000, 3))
    tp = rng.random((1500, 3))
    sv = rng.standard_normal(2000)
    out = np.zeros(len(tp))
    st = np.full(len(tp), -7, dtype=np.int32)
    rc = _shim().pacman_fe_interpolate_c(3, 3, 0xF0, _dp(sp), len(sp), _dp(sv), None, 0, None, 0,
                                         None, _dp(tp), len(tp), _dp(out), st.ctypes.data_as(_I))
    assert rc == 0
    assert np.array_equal(out, oracle.fe_nearest(3, sp, sv, tp)[0])
    assert (st == 0).all()


@pytest.mark.gpu
def test_shim_mls_matches_oracle():
    rng = np.random.default_rng(7)
    sp = rng.random((3000, 3))
    tp = rng.random((2000, 3))
    sv = np.cos(4 * sp[:, 0]) * sp[:, 1]
    out = np.zeros(len(tp))
    rc = _shim().pacman_mls_interpolate_c(3, 3, _dp(sp), len(sp), _dp(sv), _dp(tp), len(tp),
                                          _dp(out))
    assert rc == 0
    assert np.array_equal(out, oracle.mls_interpolate(3, sp, sv, tp))
