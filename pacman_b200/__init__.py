"""B200-native RBF-PUM transfer, a drop-in for PACMAN's ``pacman`` module.

``import pacman_b200 as pacman`` then ``pacman.rbf.interpolate(...)`` with the
reference's arguments (src/pybindings/bindings.cpp:38-93).  The computation
runs in hand-written sm_100a CUDA kernels behind the C ABI of
``include/pacman_b200.h``; there is no CPU fallback.
"""
from . import distributed, execspaces, fe, mls, rbf  # noqa: F401
from . import mls as MLS  # noqa: F401  (the reference's submodule name)
from ._lib import load as _load_library

__all__ = ["MLS", "distributed", "execspaces", "fe", "mls", "rbf", "initialize", "finalize",
           "library_path"]


def initialize():
    """Loads the engine (the reference initialises Kokkos here, bindings.cpp:26-30)."""
    _load_library()


def finalize():
    """No-op: device state is released with each call or plan
    (the reference finalises Kokkos here, bindings.cpp:31-35)."""


def library_path() -> str:
    from ._lib import LIB_PATH
    return LIB_PATH
