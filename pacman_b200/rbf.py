"""``pacman.rbf`` on the B200 engine.

Mirrors the reference's Python binding (src/pybindings/bindings.cpp:75-93,
src/pybindings/rbf_bindings.cpp:74-120): ``interpolate(space_dimension,
execspace, rbf_function, source_points, source_values, target_points)`` with
the same argument meaning, the same shape checks and the same exception
types, returning a float64 array of length ``len(target_points)``.

Superset keywords: ``nodes_per_cluster``, ``relative_overlap`` and
``support_radius`` (the reference's hard-coded defaults 50 / 0.15 / 0.1,
src/rbf_pum/interpolator.hxx:39-41), ``precision`` ("fp64": the reference's
unpivoted-LU algorithm; "mixed": Cholesky with the column updates of large
patches as split-integer products on the int8 tensor cores, FP64-level
accuracy, small patches in FP64 registers), multi-field ``source_values`` of
shape (N, F) with F <= 8, and CUDA torch tensors (device-resident inputs and
output, ordered on torch's current stream).
"""
from __future__ import annotations

import ctypes
import types

import numpy as np

from . import _lib
from .execspaces import _VALID as _VALID_EXEC

functions = types.SimpleNamespace(
    WENDLANDC0=0x10, WENDLANDC2=0x11, WENDLANDC4=0x12, WENDLANDC6=0x13, WENDLANDC8=0x14)

_PRECISION = {"fp64": _lib.FP64, "mixed": _lib.MIXED}


def _is_cuda_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _options(nodes_per_cluster, relative_overlap, support_radius, precision, device, stream):
    o = _lib.default_options()
    o.nodes_per_cluster = int(nodes_per_cluster)
    o.relative_overlap = float(relative_overlap)
    o.support_radius = float(support_radius)
    if precision not in _PRECISION:
        raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
    o.precision = _PRECISION[precision]
    o.device = -1 if device is None else int(device)
    o.stream = stream
    return o


def _check_shapes(space_dimension, sp_shape, sv_shape, tp_shape):
    """The reference's checks (rbf_bindings.cpp:83-104) plus dim agreement."""
    if len(sp_shape) != 2:
        raise ValueError("Source points must be a 2-d numpy array!")
    if len(tp_shape) != 2:
        raise ValueError("Target points must be a 2-d numpy array!")
    if sp_shape[1] != tp_shape[1]:
        raise ValueError(
            "Dimensions mismatch between source points and target points!\n"
            f"Provided source points dimension: {sp_shape[1]}\n"
            f"Provided target points dimension: {tp_shape[1]}\n")
    if len(sv_shape) == 0 or sp_shape[0] != sv_shape[0]:
        raise ValueError(
            "Each source point must have its corresponding value in the source values!\n"
            f"Number of source points: {sp_shape[0]}\n"
            f"Number of source values: {sv_shape[0] if len(sv_shape) else 0}\n")
    if space_dimension not in (1, 2, 3):
        raise RuntimeError("The dimension of the points can only be: 1, 2 or 3.\n")
    if sp_shape[1] != space_dimension:
        raise ValueError(
            f"points have {sp_shape[1]} coordinates but space_dimension is {space_dimension}")
    if len(sv_shape) > 2 or (len(sv_shape) == 2 and not 1 <= sv_shape[1] <= 8):
        raise ValueError("source values must have shape (N,) or (N, F) with 1 <= F <= 8")


def interpolate(space_dimension, execspace, rbf_function, source_points, source_values,
                target_points, *, nodes_per_cluster=50, relative_overlap=0.15,
                support_radius=0.1, precision="fp64", device=None, stats=None, stream=None):
    """RBF-PUM transfer of ``source_values`` from ``source_points`` to
    ``target_points``.  Returns float64 values at the targets, (M,) for 1-D
    values and (M, F) for (N, F) values; a CUDA torch tensor when the inputs
    are CUDA torch tensors.  ``stats`` (a dict) receives the call statistics;
    ``stream`` (a cudaStream_t handle) orders a host-input call on that stream."""
    lib = _lib.load()
    if int(execspace) not in _VALID_EXEC:
        raise ValueError("execspace: Serial, OpenMP, Threads, Cuda, HIP, SYCL")
    if int(rbf_function) not in vars(functions).values():
        raise ValueError(f"Unsupported RBF function selector: {int(rbf_function)}")
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
    _check_shapes(int(space_dimension), *shapes)
    n, m = shapes[0][0], shapes[2][0]
    F = 1 if len(shapes[1]) == 1 else shapes[1][1]
    out_shape = (m,) if len(shapes[1]) == 1 else (m, F)
    st = _lib.Stats()
    if on_gpu:
        import torch
        out = torch.empty(out_shape, dtype=torch.float64, device=sp.device)
        stream = torch.cuda.current_stream(sp.device).cuda_stream
        opts = _options(nodes_per_cluster, relative_overlap, support_radius, precision,
                        sp.device.index, stream)
        ptrs = (sp.data_ptr(), sv.data_ptr(), tp.data_ptr(), out.data_ptr())
    else:
        out = np.zeros(out_shape, dtype=np.float64)
        opts = _options(nodes_per_cluster, relative_overlap, support_radius, precision, device,
                        stream)
        ptrs = (sp.ctypes.data, sv.ctypes.data, tp.ctypes.data, out.ctypes.data)
    if m == 0:
        return out
    rc = lib.pacman_b200_rbf_interpolate(int(space_dimension), int(rbf_function), ptrs[0], n,
                                         ptrs[1], F, ptrs[2], m, ptrs[3], ctypes.byref(opts),
                                         ctypes.byref(st))
    _lib.raise_for(rc, "pacman.rbf.interpolate")
    if stats is not None:
        stats.update(st.as_dict())
    return out


def interpolate_batch(problems, *, nodes_per_cluster=50, relative_overlap=0.15,
                      support_radius=0.1, precision="fp64", device=None, stats=None,
                      stream=None):
    """Many independent transfers in one call (no counterpart in the
    reference, which runs one transfer per call).  ``problems`` is a sequence
    of ``(space_dimension, rbf_function, source_points, source_values,
    target_points)`` with the meaning, shapes and checks of ``interpolate``;
    all numpy or all CUDA torch tensors on one device.  The patches of every
    problem that shares (space_dimension, rbf_function) are solved together in
    one set of launches.  Returns the list of target values, each as
    ``interpolate`` returns it; ``stats`` receives the totals."""
    lib = _lib.load()
    items = list(problems)
    if not items:
        return []
    on_gpu = _is_cuda_tensor(items[0][2])
    keep, outs = [], []
    arr = (_lib.Problem * len(items))()
    dev = None
    for i, item in enumerate(items):
        if len(item) != 5:
            raise ValueError("each problem is (space_dimension, rbf_function, source_points, "
                             "source_values, target_points)")
        dim, fn, sp, sv, tp = item
        if int(fn) not in vars(functions).values():
            raise ValueError(f"Unsupported RBF function selector: {int(fn)}")
        if _is_cuda_tensor(sp) != on_gpu:
            raise ValueError("problems must be all numpy or all CUDA tensors")
        if on_gpu:
            import torch
            sp = sp.to(torch.float64).contiguous()
            if dev is None:
                dev = sp.device
            elif sp.device != dev:
                raise ValueError("all CUDA problems must be on one device")
            sv = sv.to(device=dev, dtype=torch.float64).contiguous()
            tp = tp.to(device=dev, dtype=torch.float64).contiguous()
            shapes = (tuple(sp.shape), tuple(sv.shape), tuple(tp.shape))
        else:
            sp = np.ascontiguousarray(sp, dtype=np.float64)
            sv = np.ascontiguousarray(sv, dtype=np.float64)
            tp = np.ascontiguousarray(tp, dtype=np.float64)
            shapes = (sp.shape, sv.shape, tp.shape)
        _check_shapes(int(dim), *shapes)
        n, m = shapes[0][0], shapes[2][0]
        F = 1 if len(shapes[1]) == 1 else shapes[1][1]
        out_shape = (m,) if len(shapes[1]) == 1 else (m, F)
        if on_gpu:
            import torch
            out = torch.empty(out_shape, dtype=torch.float64, device=dev)
            ptrs = (sp.data_ptr(), sv.data_ptr(), tp.data_ptr(), out.data_ptr())
        else:
            out = np.zeros(out_shape, dtype=np.float64)
            ptrs = (sp.ctypes.data, sv.ctypes.data, tp.ctypes.data, out.ctypes.data)
        keep.append((sp, sv, tp))
        outs.append(out)
        arr[i] = _lib.Problem(int(dim), int(fn), ptrs[0] if n else None, n,
                              ptrs[1] if n else None, F, ptrs[2] if m else None, m,
                              ptrs[3] if m else None)
    if on_gpu:
        import torch
        stream = torch.cuda.current_stream(dev).cuda_stream
        device = dev.index
    opts = _options(nodes_per_cluster, relative_overlap, support_radius, precision, device,
                    stream)
    st = _lib.Stats()
    rc = lib.pacman_b200_rbf_interpolate_batch(arr, len(items), ctypes.byref(opts),
                                               ctypes.byref(st))
    _lib.raise_for(rc, "pacman.rbf.interpolate_batch")
    if stats is not None:
        stats.update(st.as_dict())
    return outs


def _as_array(x):
    """(pointer, shape, kind, keep-alive) of a float64 C-contiguous view of x:
    CUDA torch tensors stay on the device, everything else becomes numpy."""
    if _is_cuda_tensor(x):
        import torch
        t = x.detach().to(torch.float64).contiguous()
        return t.data_ptr(), tuple(t.shape), "cuda", t
    a = np.ascontiguousarray(x, dtype=np.float64)
    return a.ctypes.data, a.shape, "host", a


def _empty_like_kind(kind, shape, ref):
    if kind == "cuda":
        import torch
        t = torch.zeros(shape, dtype=torch.float64, device=ref.device)
        return t.data_ptr(), t
    a = np.zeros(shape, dtype=np.float64)
    return a.ctypes.data, a


class Plan:
    """Reusable transfer plan: geometry built once, ``execute`` per field set.

    The geometry (patch radius, centre cover, membership lists) depends only
    on the points, so coupling loops that move new values over fixed meshes
    skip it after the first call.  Points, values and gradients may be numpy
    arrays or CUDA torch tensors."""

    def __init__(self, space_dimension, source_points, target_points, *, nodes_per_cluster=50,
                 relative_overlap=0.15, support_radius=0.1, precision="fp64", device=None):
        self._lib = _lib.load()
        self._h = None
        sp_ptr, sp_shape, kind, self._sp = _as_array(source_points)
        tp_ptr, tp_shape, _, self._tp = _as_array(target_points)
        _check_shapes(int(space_dimension), sp_shape, (sp_shape[0],), tp_shape)
        self.dim = int(space_dimension)
        self.n, self.m = sp_shape[0], tp_shape[0]
        if kind == "cuda" and device is None:
            device = self._sp.device.index
        opts = _options(nodes_per_cluster, relative_overlap, support_radius, precision, device,
                        None)
        h = ctypes.c_void_p()
        rc = self._lib.pacman_b200_plan_create(self.dim, sp_ptr, self.n, tp_ptr, self.m,
                                               ctypes.byref(opts), ctypes.byref(h))
        _lib.raise_for(rc, "pacman.rbf.Plan")
        self._h = h
        self.F = None

    def close(self):
        if self._h is not None and self._h.value:
            self._lib.pacman_b200_plan_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        r = ctypes.c_double()
        info = (ctypes.c_int64 * 4)()
        _lib.raise_for(self._lib.pacman_b200_plan_info(self._h, ctypes.byref(r), info))
        return dict(radius=r.value, num_patches=info[0], num_candidates=info[1],
                    src_nnz=info[2], tgt_nnz=info[3])

    def centers(self) -> np.ndarray:
        K = self.info()["num_patches"]
        out = np.zeros((K, self.dim), dtype=np.float64)
        if K:
            _lib.raise_for(self._lib.pacman_b200_plan_centers(self._h, out.ctypes.data))
        return out

    def patch_lists(self, which: str = "source"):
        inf = self.info()
        K = inf["num_patches"]
        w = 0 if which == "source" else 1
        nnz = inf["src_nnz"] if w == 0 else inf["tgt_nnz"]
        off = np.zeros(K + 1, dtype=np.int64)
        idx = np.zeros(max(nnz, 1), dtype=np.int32)
        _lib.raise_for(self._lib.pacman_b200_plan_patch_lists(self._h, w, off.ctypes.data,
                                                               idx.ctypes.data))
        return off, idx[:nnz]

    def shard(self, rank: int, world: int) -> "Plan":
        """Keeps target shard ``rank`` of ``world`` (one process per GPU, each
        with the same plan): executes then solve only the patches the shard's
        targets need and return their values, bit-identical to the unsharded
        transfer, with zeros at the other targets; the sum over the ranks is
        the whole result.  See ``pacman_b200.distributed``."""
        _lib.raise_for(self._lib.pacman_b200_plan_shard(self._h, int(rank), int(world)),
                       "pacman.rbf.Plan.shard")
        return self

    def owned_targets(self) -> np.ndarray:
        """Indices (ascending) of the targets of this plan's shard."""
        cnt = ctypes.c_int64()
        _lib.raise_for(self._lib.pacman_b200_plan_owned_targets(self._h, ctypes.byref(cnt), None))
        out = np.zeros(max(cnt.value, 1), dtype=np.int32)
        _lib.raise_for(self._lib.pacman_b200_plan_owned_targets(self._h, ctypes.byref(cnt),
                                                                out.ctypes.data))
        return out[: cnt.value]

    def local_values(self) -> np.ndarray:
        inf = self.info()
        out = np.zeros((max(inf["tgt_nnz"], 1), self.F or 1), dtype=np.float64)
        _lib.raise_for(self._lib.pacman_b200_plan_local_values(self._h, out.ctypes.data))
        return out[: inf["tgt_nnz"]]

    def patch_status(self) -> np.ndarray:
        """Per-patch status words of the last execute (int32, K entries):
        bit 1 polynomial axis dropped, 2 non-finite value, 4 non-positive
        Cholesky pivot, 8 tensor-core pipeline time-out, 16 re-solved by the
        FP64 LU."""
        K = self.info()["num_patches"]
        out = np.zeros(max(K, 1), dtype=np.int32)
        _lib.raise_for(self._lib.pacman_b200_plan_patch_status(self._h, out.ctypes.data))
        return out[:K]

    def execute(self, rbf_function, source_values, stats=None, save_for_adjoint=False,
                time_kernels=False, keep_factors=False):
        """Transfer of source_values ((N,) or (N, F)); with save_for_adjoint the
        per-patch coefficients are kept for ``adjoint``; with time_kernels the
        dominant kernel's launches are timed with CUDA events into ``stats``;
        with keep_factors (precision "mixed") the patch factorisations are kept
        by the first such execute and reused by the later ones with the same
        basis (only the polynomial block, the triangular solves and the
        evaluation run again)."""
        ptr, shape, kind, keep = _as_array(source_values)
        if shape[0] != self.n:
            raise ValueError("source values must have one row per source point")
        F = 1 if len(shape) == 1 else shape[1]
        out_ptr, out = _empty_like_kind(kind, (self.m,) if len(shape) == 1 else (self.m, F), keep)
        st = _lib.Stats()
        flags = (_lib.SAVE_FOR_ADJOINT if save_for_adjoint else 0) | (
            _lib.TIME_KERNELS if time_kernels else 0) | (_lib.KEEP_FACTORS if keep_factors else 0)
        rc = self._lib.pacman_b200_plan_execute_ex(self._h, int(rbf_function), ptr, F, out_ptr,
                                                   flags, ctypes.byref(st))
        _lib.raise_for(rc, "pacman.rbf.Plan.execute")
        self.F = F
        self._vector = len(shape) == 1
        if stats is not None:
            stats.update(st.as_dict())
        return out

    def adjoint(self, grad_target_values, values=True, targets=True):
        """Transpose of the last execute(save_for_adjoint=True): returns
        (d<G, out>/d source_values, d<G, out>/d target_points) for the upstream
        gradient G (same shape as that execute's output); either may be None."""
        ptr, shape, kind, keep = _as_array(grad_target_values)
        F = self.F
        vshape = (self.n,) if self._vector else (self.n, F)
        gv_ptr, gv = _empty_like_kind(kind, vshape, keep) if values else (None, None)
        gt_ptr, gt = _empty_like_kind(kind, (self.m, self.dim), keep) if targets else (None, None)
        rc = self._lib.pacman_b200_plan_adjoint(self._h, ptr, gv_ptr, gt_ptr)
        _lib.raise_for(rc, "pacman.rbf.Plan.adjoint")
        return gv, gt
