"""ctypes binding of libpacman_b200.so (the C ABI of include/pacman_b200.h).

The shared library is loaded from this package directory.  There is no CPU
fallback: if the library is missing or cannot be loaded, every entry point
raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpacman_b200.so")

OK = 0
ERR_INVALID = -1
ERR_DIMENSION = -2
ERR_CUDA = -3
ERR_NOMEM = -4
ERR_DEGENERATE = -5
ERR_LIMIT = -6

FP64 = 0
MIXED = 1
SAVE_FOR_ADJOINT = 1
TIME_KERNELS = 2
KEEP_FACTORS = 4

_lock = threading.Lock()
_lib = None


class Options(ctypes.Structure):
    _fields_ = [
        ("nodes_per_cluster", ctypes.c_int32),
        ("relative_overlap", ctypes.c_double),
        ("support_radius", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("stream", ctypes.c_void_p),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_double),
        ("num_candidates", ctypes.c_int64),
        ("num_patches", ctypes.c_int64),
        ("sum_n", ctypes.c_int64),
        ("sum_m", ctypes.c_int64),
        ("max_n", ctypes.c_int64),
        ("patches_fp32", ctypes.c_int64),
        ("patches_fp64", ctypes.c_int64),
        ("patches_fallback", ctypes.c_int64),
        ("dropped_axis_patches", ctypes.c_int64),
        ("ms_geometry", ctypes.c_double),
        ("ms_solve", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("kernel_launches", ctypes.c_int64),
        ("ms_factor", ctypes.c_double),
        ("factor_flops", ctypes.c_double),
        ("ms_update", ctypes.c_double),
        ("update_flops", ctypes.c_double),
        ("update_launches", ctypes.c_int64),
        ("factors_reused", ctypes.c_int64),
        ("ms_update_i8", ctypes.c_double),
        ("update_flops_i8", ctypes.c_double),
        ("update_launches_i8", ctypes.c_int64),
        ("ms_update_f64", ctypes.c_double),
        ("update_flops_f64", ctypes.c_double),
        ("update_launches_f64", ctypes.c_int64),
        ("host_syncs", ctypes.c_int64),
        ("mma_products_i8", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Problem(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("rbf_function", ctypes.c_int32),
        ("source_points", ctypes.c_void_p),
        ("n_source", ctypes.c_int64),
        ("source_values", ctypes.c_void_p),
        ("n_fields", ctypes.c_int32),
        ("target_points", ctypes.c_void_p),
        ("n_target", ctypes.c_int64),
        ("target_values", ctypes.c_void_p),
    ]


# name -> (restype, argtypes); every symbol declared in include/pacman_b200.h.
_VP = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "pacman_b200_options_init": (None, [ctypes.POINTER(Options)]),
    "pacman_b200_rbf_interpolate": (ctypes.c_int, [
        ctypes.c_int32, ctypes.c_int32, _VP, ctypes.c_int64, _VP, ctypes.c_int32, _VP,
        ctypes.c_int64, _VP, ctypes.POINTER(Options), ctypes.POINTER(Stats)]),
    "pacman_b200_rbf_interpolate_batch": (ctypes.c_int, [
        ctypes.POINTER(Problem), ctypes.c_int32, ctypes.POINTER(Options),
        ctypes.POINTER(Stats)]),
    "pacman_b200_plan_create": (ctypes.c_int, [
        ctypes.c_int32, _VP, ctypes.c_int64, _VP, ctypes.c_int64, ctypes.POINTER(Options),
        ctypes.POINTER(_VP)]),
    "pacman_b200_plan_execute": (ctypes.c_int, [
        _VP, ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.POINTER(Stats)]),
    "pacman_b200_plan_destroy": (None, [_VP]),
    "pacman_b200_plan_execute_ex": (ctypes.c_int, [
        _VP, ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_uint32, ctypes.POINTER(Stats)]),
    "pacman_b200_plan_adjoint": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "pacman_b200_plan_info": (ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_int64)]),
    "pacman_b200_plan_centers": (ctypes.c_int, [_VP, _VP]),
    "pacman_b200_plan_patch_lists": (ctypes.c_int, [_VP, ctypes.c_int32, _VP, _VP]),
    "pacman_b200_plan_local_values": (ctypes.c_int, [_VP, _VP]),
    "pacman_b200_plan_patch_status": (ctypes.c_int, [_VP, _VP]),
    "pacman_b200_plan_shard": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32]),
    "pacman_b200_fe_interpolate": (ctypes.c_int, [
        ctypes.c_int32, ctypes.c_int32, _VP, ctypes.c_int64, _VP, _VP, ctypes.c_int64, _VP, _VP,
        ctypes.POINTER(Options)]),
    "pacman_b200_mls_interpolate": (ctypes.c_int, [
        ctypes.c_int32, _VP, ctypes.c_int64, _VP, _VP, ctypes.c_int64, _VP,
        ctypes.POINTER(Options)]),
    "pacman_b200_plan_owned_targets": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), _VP]),
    "pacman_b200_patch_radius_noalloc": (ctypes.c_int, [
        ctypes.c_int32, _VP, ctypes.c_int64, ctypes.c_int32, _VP, _VP]),
    "pacman_b200_last_error": (ctypes.c_char_p, []),
    "pacman_b200_abi_version": (ctypes.c_int32, []),
}


def load():
    """Loads the library once (raises if it is missing: no fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m pacman_b200.build` "
                "(the B200 engine has no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    return load().pacman_b200_last_error().decode()


def default_options() -> Options:
    o = Options()
    load().pacman_b200_options_init(ctypes.byref(o))
    return o


def raise_for(rc: int, what: str = "pacman_b200") -> None:
    """Maps a negative return code to the reference's exception types
    (std::invalid_argument -> ValueError, std::runtime_error -> RuntimeError)."""
    if rc == OK:
        return
    msg = f"{what}: {last_error()}"
    if rc == ERR_INVALID:
        raise ValueError(msg)
    if rc == ERR_NOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)
