"""gg_locate_noalloc: point location for callers that cannot allocate device memory.

Some hosts of this library cannot call cudaMalloc: a process whose device memory is all
handed out by its own allocator or a fixed arena, and real-time drivers that forbid
allocation once they run.  They pass the points and the output buffers they own; the
entry point keeps its counting-sort scratch in a fixed device array.  This test gives it
device buffers (allocated here, by the test, as such a caller would own them), calls it
twice in a row and checks both results against the existing entry point, gg_locate:
cells bit-exact, and offsets/order equal to the stable per-element order of those cells.
It runs last (file name) so that a failure here leaves every other test already run,
and it passes both alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from gale_b200 import abi, workloads
from gale_b200.stokes import MaterialViscosity, Mesh, RheologyMaterial, StokesProblem

pytestmark = pytest.mark.gpu


def reference_cells(mesh, coords):
    """Cells from the existing entry point gg_locate (through a handle)."""
    G = StokesProblem(mesh)
    G.set_materials([RheologyMaterial([MaterialViscosity(1.0)])])
    G.set_points(coords)
    cell = np.empty(coords.shape[0], dtype=np.uint32)
    rc = G.lib.gg_locate(G.h, cell.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert rc in (abi.GG_OK, abi.GG_ERR_OUT_OF_DOMAIN)
    return cell


def call_noalloc(lib, mesh, coords, torch):
    n = coords.shape[0]
    nel = int(np.prod([mesh.elements[d] for d in range(mesh.dim)]))
    d_coords = torch.from_numpy(coords).cuda()
    d_cell = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_off = torch.full((nel + 1,), -1, dtype=torch.int32, device="cuda")
    d_order = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    outside = C.c_int64(-1)
    msg = C.c_char_p()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = lib.gg_locate_noalloc(C.byref(mesh), n, d_coords.data_ptr(), d_cell.data_ptr(), d_off.data_ptr(),
                               d_order.data_ptr(), C.byref(outside), None, C.byref(msg))
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    return (rc, d_cell.cpu().numpy().view(np.uint32), d_off.cpu().numpy(), d_order.cpu().numpy(),
            outside.value, (msg.value or b"").decode(), free_before - free_after)


@pytest.mark.parametrize("make", [lambda: workloads.creep_3d(n=16), lambda: workloads.sinker_2d(n=64)],
                         ids=["3d", "2d"])
def test_noalloc_matches_gg_locate_twice(make):
    torch = pytest.importorskip("torch")
    w = make()
    lib = abi.load_library()
    expect = reference_cells(w.mesh, w.coords)
    order_expect = np.argsort(expect, kind="stable").astype(np.int32)
    nel = w.nel
    off_expect = np.concatenate([[0], np.cumsum(np.bincount(expect, minlength=nel))]).astype(np.int32)
    for k in range(2):  # the second call reuses the scratch the first one left behind
        rc, cell, off, order, outside, msg, grown = call_noalloc(lib, w.mesh, w.coords, torch)
        assert rc == abi.GG_OK, msg
        if k == 1:
            assert grown == 0  # the device's free memory is the same after the call
        assert outside == 0
        assert np.array_equal(cell, expect)
        assert np.array_equal(off, off_expect)
        assert np.array_equal(order, order_expect)


def test_noalloc_outside_points_and_limits():
    torch = pytest.importorskip("torch")
    lib = abi.load_library()
    mesh = Mesh(2, (32, 32))
    rng = np.random.default_rng(4)
    x = np.ascontiguousarray(rng.uniform(-0.05, 1.05, size=(5000, 2)))
    expect = reference_cells(mesh, x)
    for _ in range(2):
        rc, cell, off, order, outside, msg, grown = call_noalloc(lib, mesh, x, torch)
        assert rc == abi.GG_ERR_OUT_OF_DOMAIN
        assert grown == 0
        assert np.array_equal(cell, expect)
        assert outside == int((expect == 32 * 32).sum()) > 0
        inside = expect < 32 * 32
        assert off[-1] == inside.sum()
        assert np.array_equal(order[:off[-1]], np.argsort(np.where(inside, expect, 1 << 30), kind="stable")[:off[-1]])
        assert (order[off[-1]:] == -1).all()  # past the last element: the caller's contents
    # sizes beyond the fixed scratch are rejected with a message, nothing launched
    big = Mesh(2, (2048, 1024))
    msg = C.c_char_p()
    rc = lib.gg_locate_noalloc(C.byref(big), 10, 1, 1, 1, 1, None, None, C.byref(msg))
    assert rc == abi.GG_ERR_INVALID and b"1048576" in msg.value
