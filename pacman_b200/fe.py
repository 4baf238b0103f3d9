"""``pacman.fe`` on the B200 engine: the point-based finite-element method.

Mirrors the reference's binding ``pacman.fe.interpolate(space_dimension,
execspace, method, source_points, source_values, conn_val, conn_off,
cell_types, target_points)`` (src/pybindings/bindings.cpp:95-107,
src/pybindings/fe_bindings.cpp:134-180), returning ``(target_values,
target_status)``, for ``methods.NEAREST_NEAREST``: every target takes its
nearest source's value (lowest source index on ties), and the status stays
0 (OUTSIDE), as the reference's FTNearest leaves it.  The mesh-based methods
(INTERP_*) need the element connectivity and are not part of this engine:
they raise ``ValueError``.
"""
from __future__ import annotations

import ctypes
import types

import numpy as np

from . import _lib
from .execspaces import _VALID as _VALID_EXEC
from .rbf import _is_cuda_tensor

methods = types.SimpleNamespace(
    NEAREST_NEAREST=0xF0, INTERP_CLAMP=0xF1, INTERP_NEAREST=0xF2, INTERP_ZEROFILL=0xF3,
    INTERP_EXTRAP=0xF4)


def interpolate(space_dimension, execspace, method, source_points, source_values, conn_val,
                conn_off, cell_types, target_points, *, device=None, stream=None):
    """Finite-element transfer with the reference's arguments and checks
    (fe_bindings.cpp:144-164); conn_val, conn_off and cell_types are accepted
    and unused by NEAREST_NEAREST.  numpy inputs give numpy outputs; CUDA torch
    tensors give CUDA tensors, ordered on torch's current stream."""
    lib = _lib.load()
    if int(execspace) not in _VALID_EXEC:
        raise ValueError("execspace: Serial, OpenMP, Threads, Cuda, HIP, SYCL")
    on_gpu = _is_cuda_tensor(source_points)
    if on_gpu:
        import torch
        sp = source_points.to(torch.float64).contiguous()
        sv = source_values.to(device=sp.device, dtype=torch.float64).contiguous()
        tp = target_points.to(device=sp.device, dtype=torch.float64).contiguous()
        shapes = (tuple(sp.shape), tuple(sv.shape), tuple(tp.shape))
    else:
        sp = np.ascontiguousarray(source_points, dtype=np.float64)
        sv = np.ascontiguousarray(source_values, dtype=np.float64)
        tp = np.ascontiguousarray(target_points, dtype=np.float64)
        shapes = (sp.shape, sv.shape, tp.shape)
    if len(shapes[0]) != 2:
        raise ValueError("Source points must be a 2-d numpy array!")
    if len(shapes[2]) != 2:
        raise ValueError("Target points must be a 2-d numpy array!")
    if shapes[0][1] != shapes[2][1]:
        raise ValueError(
            "Dimensions mismatch between source points and target points!\n"
            f"Provided source points dimension: {shapes[0][1]}\n"
            f"Provided target points dimension: {shapes[2][1]}\n")
    if len(shapes[1]) == 0 or shapes[0][0] != shapes[1][0]:
        raise ValueError(
            "Each source point must have its corresponding value in the source values!\n"
            f"Number of source points: {shapes[0][0]}\n"
            f"Number of source values: {shapes[1][0] if len(shapes[1]) else 0}\n")
    if int(space_dimension) not in (1, 2, 3):
        raise RuntimeError("The dimension of the points can only be: 1, 2 or 3.\n")
    if shapes[0][1] != int(space_dimension):
        raise ValueError(
            f"points have {shapes[0][1]} coordinates but space_dimension is {space_dimension}")
    n, m = shapes[0][0], shapes[2][0]
    o = _lib.default_options()
    if on_gpu:
        import torch
        out = torch.zeros(m, dtype=torch.float64, device=sp.device)
        status = torch.zeros(m, dtype=torch.int32, device=sp.device)
        o.device = sp.device.index
        o.stream = torch.cuda.current_stream(sp.device).cuda_stream
        ptrs = (sp.data_ptr(), sv.data_ptr(), tp.data_ptr(), out.data_ptr(), status.data_ptr())
    else:
        out = np.zeros(m, dtype=np.float64)
        status = np.zeros(m, dtype=np.int32)
        o.device = -1 if device is None else int(device)
        o.stream = stream
        ptrs = (sp.ctypes.data, sv.ctypes.data, tp.ctypes.data, out.ctypes.data,
                status.ctypes.data)
    if m == 0:
        return out, status
    rc = lib.pacman_b200_fe_interpolate(int(space_dimension), int(method),
                                        ptrs[0] if n else None, n, ptrs[1] if n else None,
                                        ptrs[2], m, ptrs[3], ptrs[4], ctypes.byref(o))
    _lib.raise_for(rc, "pacman.fe.interpolate")
    return out, status
