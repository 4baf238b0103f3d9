"""``pacman.MLS`` on the B200 engine: moving least squares transfer.

Mirrors the reference's binding ``pacman.MLS.interpolate(space_dimension,
execspace, source_points, source_values, target_points)``
(src/pybindings/bindings.cpp:124-133, src/pybindings/mls_bindings.cpp), the
same shape checks and messages, returning the target values.  The reference
calls ArborX's MovingLeastSquares with its defaults; this engine computes the
same fit (K = 3, 6, 10 nearest sources in 1D, 2D, 3D, Wendland C0 weights, a
quadratic least-squares polynomial evaluated at the target) in one CUDA
kernel, behind ``pacman_b200_mls_interpolate`` of ``include/pacman_b200.h``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .execspaces import _VALID as _VALID_EXEC
from .rbf import _is_cuda_tensor


def interpolate(space_dimension, execspace, source_points, source_values, target_points, *,
                device=None, stream=None):
    """One scalar field from the sources to the targets.  numpy inputs give a
    numpy output; CUDA torch tensors give a CUDA tensor, ordered on torch's
    current stream."""
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
    # mls_bindings.cpp: Interpolate's checks, in its order.
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
        o.device = sp.device.index
        o.stream = torch.cuda.current_stream(sp.device).cuda_stream
        ptrs = (sp.data_ptr(), sv.data_ptr(), tp.data_ptr(), out.data_ptr())
    else:
        out = np.zeros(m, dtype=np.float64)
        o.device = -1 if device is None else int(device)
        o.stream = stream
        ptrs = (sp.ctypes.data, sv.ctypes.data, tp.ctypes.data, out.ctypes.data)
    if m == 0:
        return out
    rc = lib.pacman_b200_mls_interpolate(int(space_dimension), ptrs[0] if n else None, n,
                                         ptrs[1] if n else None, ptrs[2], m, ptrs[3],
                                         ctypes.byref(o))
    _lib.raise_for(rc, "pacman.MLS.interpolate")
    return out
