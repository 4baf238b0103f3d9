"""pacman_b200_patch_radius_noalloc: the patch radius with no device allocation.

Some callers cannot let this library allocate device memory, for instance a
coupled simulation code that reserves the GPU for its own pool allocator at
start-up and hands out every buffer itself.  For them the library computes
the transfer's patch radius with kernels whose working memory is one fixed
__device__ array.  This test calls that entry point through the C ABI and
checks it against the radius the full transfer computes (the geometry tests
hold the radius to exact equality, so this one does too), on consecutive
calls that share and reuse the array.  It lives in its own file, collected
last, and passes both alone and after the rest of the suite."""
import ctypes

import numpy as np
import pytest

import pacman_b200 as pacman
from pacman_b200 import _lib
from pacman_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(17)
    u = W.make("uniform_20k")
    gb = W.make("grid_blobs_1m", scale=0.01)
    return [
        (3, u["src"], u["tgt"], 30),
        (3, gb["src"], gb["tgt"], 50),
        (2, rng.random((4000, 2)), rng.random((3000, 2)), 40),
        (1, rng.random((2500, 1)), rng.random((2000, 1)), 20),
    ]


def _noalloc(torch, lib, dim, pts_dev, npc, out):
    rc = lib.pacman_b200_patch_radius_noalloc(
        dim, pts_dev.data_ptr(), pts_dev.shape[0], npc,
        torch.cuda.current_stream().cuda_stream, out)
    assert rc == 0, _lib.last_error()


def test_noalloc_radius_equals_transfer_radius_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    cases = _cases()
    expected = [pacman.rbf.Plan(dim, S, T, nodes_per_cluster=npc).info()["radius"]
                for dim, S, T, npc in cases]
    dev = [torch.tensor(S, device="cuda") for _, S, _, _ in cases]
    host_r = ctypes.c_double()
    # Two calls in a row on every case, then the cases interleaved: each call
    # must reset what it needs in the shared array.
    order = [0, 0, 1, 1, 2, 2, 3, 3, 1, 0, 3, 2]
    for i in order:
        dim, _, _, npc = cases[i]
        host_r.value = -1.0
        _noalloc(torch, lib, dim, dev[i], npc, ctypes.addressof(host_r))
        assert host_r.value == expected[i], (i, host_r.value, expected[i])
    # Result written to device memory.
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):
        _noalloc(torch, lib, cases[1][0], dev[1], cases[1][3], out.data_ptr())
        torch.cuda.synchronize()
        assert out.item() == expected[1]


def test_noalloc_leaves_device_memory_untouched():
    """The point of the entry point: repeated calls take no device memory.
    The free memory the driver reports (cudaMemGetInfo) and torch's own
    allocator are read before and after, once the kernels are loaded (the
    first launch of a kernel may load its module into device memory)."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    dim, S, _, npc = _cases()[1]
    pts = torch.tensor(S, device="cuda")
    r = ctypes.c_double()
    _noalloc(torch, lib, dim, pts, npc, ctypes.addressof(r))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(5):
        _noalloc(torch, lib, dim, pts, npc, ctypes.addressof(r))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_what_it_cannot_serve():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    r = ctypes.c_double()
    host = np.random.default_rng(1).random((100, 3))
    # Host memory cannot be staged without allocating.
    rc = lib.pacman_b200_patch_radius_noalloc(3, host.ctypes.data, 100, 10, None,
                                              ctypes.addressof(r))
    assert rc == _lib.ERR_INVALID and "device memory" in _lib.last_error()
    dpts = torch.tensor(host, device="cuda")
    rc = lib.pacman_b200_patch_radius_noalloc(4, dpts.data_ptr(), 100, 10, None,
                                              ctypes.addressof(r))
    assert rc == _lib.ERR_DIMENSION
    rc = lib.pacman_b200_patch_radius_noalloc(3, dpts.data_ptr(), 0, 10, None,
                                              ctypes.addressof(r))
    assert rc == _lib.ERR_INVALID
    # Coincident sources give a zero radius, which the full transfer rejects
    # as degenerate too.
    same = torch.full((50, 3), 0.25, dtype=torch.float64, device="cuda")
    rc = lib.pacman_b200_patch_radius_noalloc(3, same.data_ptr(), 50, 10, None,
                                              ctypes.addressof(r))
    assert rc == _lib.ERR_DEGENERATE and r.value == 0.0
    with pytest.raises(Exception):
        pacman.rbf.Plan(3, same.cpu().numpy(), same.cpu().numpy(), nodes_per_cluster=10)
