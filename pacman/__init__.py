"""``import pacman`` on the B200 engine.

PACMAN's Python callers import the pybind11 module ``pacman`` and call
``pacman.rbf.interpolate(space_dimension, execspace, rbf_function,
source_points, source_values, target_points)`` with the constants of
``pacman.execspaces`` and ``pacman.rbf.functions``, after
``pacman.initialize()`` (src/pybindings/bindings.cpp:17-93).  This package
gives them the same names over ``pacman_b200``, so such a caller (the
reference's tests/test_rbf-pum.py, for one) runs unchanged once this
directory is on ``sys.path``.  ``pacman.fe.interpolate`` serves the
point-based method NEAREST_NEAREST; ``pacman.MLS.interpolate`` the moving
least squares transfer.  Nothing here computes: every call goes
to the CUDA engine behind ``include/pacman_b200.h``.
"""
from pacman_b200 import MLS, execspaces, fe, finalize, initialize, rbf  # noqa: F401

__all__ = ["MLS", "execspaces", "fe", "finalize", "initialize", "rbf"]
