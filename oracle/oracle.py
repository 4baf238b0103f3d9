"""ctypes front end of the C oracle (test infrastructure only).

The C library restates PACMAN's RBF-PUM algorithm (src/rbf_pum/) in FP64;
see rbf_pum_oracle.c for the per-function reference citations.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_rbfpum.so")
_lib = None
_lock = threading.Lock()

_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def ensure_built() -> str:
    """Compile the oracle with its Makefile if the shared library is missing."""
    src = os.path.join(_HERE, "rbf_pum_oracle.c")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        ensure_built()
        lib = ctypes.CDLL(_LIB_PATH)
        lib.orc_build.argtypes = [ctypes.c_int, _f64p, ctypes.c_int64, _f64p, ctypes.c_int64,
                                  ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_void_p)]
        lib.orc_build.restype = ctypes.c_int
        lib.orc_free.argtypes = [ctypes.c_void_p]
        lib.orc_radius.argtypes = [ctypes.c_void_p]
        lib.orc_radius.restype = ctypes.c_double
        for f in ("orc_num_patches", "orc_num_candidates", "orc_src_nnz", "orc_tgt_nnz"):
            getattr(lib, f).argtypes = [ctypes.c_void_p]
            getattr(lib, f).restype = ctypes.c_int64
        lib.orc_centers.argtypes = [ctypes.c_void_p, _f64p]
        lib.orc_src_csr.argtypes = [ctypes.c_void_p, _i64p, _i32p]
        lib.orc_tgt_csr.argtypes = [ctypes.c_void_p, _i64p, _i32p]
        lib.orc_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _f64p,
                                  ctypes.c_int, ctypes.c_int64, _f64p, _f64p, _i64p,
                                  ctypes.c_int64, _i64p, _i32p]
        lib.orc_solve.restype = ctypes.c_int
        lib.orc_weight_sums.argtypes = [ctypes.c_void_p, _f64p]
        lib.orc_poly_dropped.argtypes = [ctypes.c_void_p, _i32p]
        lib.orc_poly_dropped.restype = ctypes.c_int
        lib.orc_wendland.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.orc_wendland.restype = ctypes.c_double
        lib.orc_set_threads.argtypes = [ctypes.c_int]
        lib.orc_set_threads.restype = ctypes.c_int
        lib.orc_last_error.restype = ctypes.c_char_p
        lib.orc_fe_nearest.argtypes = [ctypes.c_int, _f64p, ctypes.c_int64, _f64p, _f64p,
                                       ctypes.c_int64, _f64p, _i32p]
        lib.orc_fe_nearest.restype = ctypes.c_int
        lib.orc_mls_interpolate.argtypes = [ctypes.c_int, _f64p, ctypes.c_int64, _f64p, _f64p,
                                            ctypes.c_int64, _f64p, _i32p, ctypes.c_int]
        lib.orc_mls_interpolate.restype = ctypes.c_int
        _lib = lib
        return lib


def _ptr(a, t=_f64p):
    return a.ctypes.data_as(t)


def set_threads(n: int) -> int:
    """Set the OpenMP thread count of the oracle; returns the count in use."""
    return _load().orc_set_threads(int(n))


def wendland(basis: int, r: float, rho: float) -> float:
    return _load().orc_wendland(int(basis), float(r), float(rho))


class OraclePlan:
    """Geometry of one transfer: radius, centres and patch membership lists."""

    def __init__(self, dim, src, tgt, nodes_per_cluster=50, relative_overlap=0.15,
                 brute_force=False):
        lib = _load()
        self.dim = int(dim)
        self.src = np.ascontiguousarray(src, dtype=np.float64).reshape(-1, self.dim)
        self.tgt = np.ascontiguousarray(tgt, dtype=np.float64).reshape(-1, self.dim)
        h = ctypes.c_void_p()
        rc = lib.orc_build(self.dim, _ptr(self.src), self.src.shape[0], _ptr(self.tgt),
                           self.tgt.shape[0], int(nodes_per_cluster), float(relative_overlap),
                           int(bool(brute_force)), ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle build failed ({rc}): {lib.orc_last_error().decode()}")
        self._h = h
        self._lib = lib

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.orc_free(h)
            self._h = None

    @property
    def radius(self) -> float:
        return self._lib.orc_radius(self._h)

    @property
    def num_patches(self) -> int:
        return self._lib.orc_num_patches(self._h)

    @property
    def num_candidates(self) -> int:
        return self._lib.orc_num_candidates(self._h)

    def centers(self) -> np.ndarray:
        out = np.empty((self.num_patches, self.dim), dtype=np.float64)
        self._lib.orc_centers(self._h, _ptr(out))
        return out

    def src_csr(self):
        K = self.num_patches
        off = np.empty(K + 1, dtype=np.int64)
        idx = np.empty(max(self._lib.orc_src_nnz(self._h), 1), dtype=np.int32)
        self._lib.orc_src_csr(self._h, _ptr(off, _i64p), _ptr(idx, _i32p))
        return off, idx[: off[-1]]

    def tgt_csr(self):
        K = self.num_patches
        off = np.empty(K + 1, dtype=np.int64)
        idx = np.empty(max(self._lib.orc_tgt_nnz(self._h), 1), dtype=np.int32)
        self._lib.orc_tgt_csr(self._h, _ptr(off, _i64p), _ptr(idx, _i32p))
        return off, idx[: off[-1]]

    def weight_sums(self) -> np.ndarray:
        out = np.empty(self.tgt.shape[0], dtype=np.float64)
        self._lib.orc_weight_sums(self._h, _ptr(out))
        return out

    def poly_dropped(self) -> np.ndarray:
        """Per patch: does its polynomial block drop an axis (bool, K)."""
        out = np.zeros(max(self.num_patches, 1), dtype=np.int32)
        rc = self._lib.orc_poly_dropped(self._h, _ptr(out, _i32p))
        if rc != 0:
            raise RuntimeError(f"oracle poly_dropped failed ({rc})")
        return out[: self.num_patches].astype(bool)

    def solve(self, basis, values, support_radius=0.1, patch_list=None, want_local=False):
        """Returns (out[m, F] or out[m], local or None, stats dict)."""
        vals = np.ascontiguousarray(values, dtype=np.float64)
        squeeze = vals.ndim == 1
        vals2 = vals.reshape(vals.shape[0], -1)
        F = vals2.shape[1]
        m = self.tgt.shape[0]
        out = np.zeros((m, F), dtype=np.float64)
        local = None
        if want_local:
            local = np.zeros((max(self._lib.orc_tgt_nnz(self._h), 1), F), dtype=np.float64)
        stats = np.zeros(8, dtype=np.int64)
        dropped = np.zeros(max(self.num_patches, 1), dtype=np.int32)
        pl = None
        npl = 0
        if patch_list is not None:
            pl = np.ascontiguousarray(patch_list, dtype=np.int64)
            npl = pl.shape[0]
        rc = self._lib.orc_solve(self._h, int(basis), float(support_radius), _ptr(vals2), F, F,
                                 _ptr(out), _ptr(local) if local is not None else None,
                                 _ptr(pl, _i64p) if pl is not None else None, npl,
                                 _ptr(stats, _i64p), _ptr(dropped, _i32p))
        if rc != 0:
            raise RuntimeError(f"oracle solve failed ({rc}): {self._lib.orc_last_error().decode()}")
        st = dict(dropped_axis_patches=int(stats[0]), sum_n3=int(stats[1]), max_n=int(stats[2]),
                  sum_n=int(stats[3]), sum_m=int(stats[4]),
                  dropped=dropped[: self.num_patches].astype(bool))
        if local is not None:
            local = local[: self._lib.orc_tgt_nnz(self._h)]
        return (out[:, 0] if squeeze else out), local, st


def build(dim, src, tgt, nodes_per_cluster=50, relative_overlap=0.15, brute_force=False):
    return OraclePlan(dim, src, tgt, nodes_per_cluster, relative_overlap, brute_force)


def interpolate(dim, basis, src, values, tgt, nodes_per_cluster=50, relative_overlap=0.15,
                support_radius=0.1):
    plan = build(dim, src, tgt, nodes_per_cluster, relative_overlap)
    out, _, _ = plan.solve(basis, values, support_radius)
    return out


def fe_nearest(dim, src, values, tgt):
    """NEAREST_NEAREST finite-element transfer (FTNearest.hpp:27-56): (values
    at the targets, nearest source index or -1)."""
    lib = _load()
    src = np.ascontiguousarray(src, dtype=np.float64).reshape(-1, dim)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64).reshape(-1, dim)
    vals = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    out = np.zeros(tgt.shape[0], dtype=np.float64)
    idx = np.zeros(max(tgt.shape[0], 1), dtype=np.int32)
    rc = lib.orc_fe_nearest(int(dim), _ptr(src) if src.size else None, src.shape[0],
                            _ptr(vals) if vals.size else None, _ptr(tgt) if tgt.size else None,
                            tgt.shape[0], _ptr(out) if out.size else None, _ptr(idx, _i32p))
    if rc != 0:
        raise RuntimeError(f"oracle fe_nearest failed ({rc}): {lib.orc_last_error().decode()}")
    return out, idx[: tgt.shape[0]]


def mls_interpolate(dim, src, values, tgt, with_sweeps=False, knn="auto"):
    """Moving least squares transfer (src/mls/interpolator.hpp:49-77 over
    ArborX's MovingLeastSquares defaults): values at the targets, and with
    ``with_sweeps`` the Jacobi sweep count of each target.  ``knn``: "brute"
    (every source per target), "grid" (a cell grid) or "auto" (the grid from
    4,096 sources on); the neighbours, and so the values, are the same."""
    lib = _load()
    src = np.ascontiguousarray(src, dtype=np.float64).reshape(-1, dim)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64).reshape(-1, dim)
    vals = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    out = np.zeros(tgt.shape[0], dtype=np.float64)
    sw = np.zeros(max(tgt.shape[0], 1), dtype=np.int32)
    rc = lib.orc_mls_interpolate(int(dim), _ptr(src) if src.size else None, src.shape[0],
                                 _ptr(vals) if vals.size else None,
                                 _ptr(tgt) if tgt.size else None, tgt.shape[0],
                                 _ptr(out) if out.size else None, _ptr(sw, _i32p),
                                 {"auto": 0, "brute": 1, "grid": 2}[knn])
    if rc != 0:
        raise RuntimeError(f"oracle mls_interpolate failed ({rc}): {lib.orc_last_error().decode()}")
    return (out, sw[: tgt.shape[0]]) if with_sweeps else out
