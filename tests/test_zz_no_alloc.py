"""galphaEdgeListNoAlloc: the allocation-free edge numbering, called through
the C ABI on device buffers and checked against the edge list that the
handle entry points (galphaTriangulate + galphaComputeResident) return for
the same mesh, which the CPU oracle's edge numbering pins in turn.  Integer
output, so the tolerance is zero.

Two meshes, three calls in a row (A, A, B): the second call shows that the
kernel leaves its shared scratch zeroed, the third that a different tile
count reuses it correctly.
"""
import ctypes

import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_TRIS = 67108864


def _lib():
    L = G.load()
    f = L.galphaEdgeListNoAlloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    L.galphaLastError.restype = ctypes.c_char_p
    return L


def _mesh(engine, n, seed, fbo):
    pts = D.uniform_points(n, seed)
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=fbo))
    al = engine.alpha_resident()
    want = np.stack([al["edge_list"]["tIndex"], al["edge_list"]["vOpp"]], axis=1).astype(np.int32)
    # the CPU oracle numbers the same triangle array's edges identically
    ref = O.alpha(pts, dt.vtx, dt.tri)["edge"]
    np.testing.assert_array_equal(want, ref[:, 5:7].astype(np.int32))
    return dt.triangles.copy(), want


def _no_alloc(L, torch, tris, cap):
    stream = torch.cuda.current_stream()
    d_tris = torch.from_numpy(tris.view(np.int32).reshape(-1).copy()).cuda()
    d_edges = torch.full((cap, 2), -7, dtype=torch.int32, device="cuda")
    d_n = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    rc = L.galphaEdgeListNoAlloc(d_tris.data_ptr(), len(tris), d_edges.data_ptr(), cap, d_n.data_ptr(),
                                 stream.cuda_stream)
    assert rc == 0, L.galphaLastError()
    torch.cuda.synchronize()
    n = int(d_n.item())
    return n, d_edges[:max(0, min(n, cap))].cpu().numpy()


def test_edge_list_no_alloc_matches_handle_path(engine):
    import torch

    L = _lib()
    tris_a, want_a = _mesh(engine, 200000, 11, 2048)
    tris_b, want_b = _mesh(engine, 3000, 12, 512)
    for tris, want in ((tris_a, want_a), (tris_a, want_a), (tris_b, want_b)):
        n, got = _no_alloc(L, torch, tris, len(want) + 16)
        assert n == len(want)
        np.testing.assert_array_equal(got, want)


def test_edge_list_no_alloc_capacity_and_limits(engine):
    import torch

    L = _lib()
    tris, want = _mesh(engine, 5000, 13, 512)
    # a short output buffer: the count is still exact, the prefix is written
    n, got = _no_alloc(L, torch, tris, 100)
    assert n == len(want)
    np.testing.assert_array_equal(got, want[:100])
    # more triangles than the fixed scratch covers: rejected before any launch
    rc = L.galphaEdgeListNoAlloc(ctypes.c_void_p(256), MAX_TRIS + 1, ctypes.c_void_p(256), 0,
                                 ctypes.c_void_p(256), None)
    assert rc == -1  # GPUDT_ERR_ARG
    assert b"scratch limit" in L.galphaLastError()
    # the call after a rejected one still works
    n, got = _no_alloc(L, torch, tris, len(want))
    assert n == len(want)
    np.testing.assert_array_equal(got, want)


def test_edge_list_no_alloc_allocates_nothing(engine):
    """Free device memory is the same before and after calls (all buffers
    made beforehand, the first call's set-up done)."""
    import torch

    L = _lib()
    tris, want = _mesh(engine, 50000, 14, 1024)
    d_tris = torch.from_numpy(tris.view(np.int32).reshape(-1).copy()).cuda()
    d_edges = torch.empty((len(want), 2), dtype=torch.int32, device="cuda")
    d_n = torch.empty((1,), dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    args = (d_tris.data_ptr(), len(tris), d_edges.data_ptr(), len(want), d_n.data_ptr(), s)
    assert L.galphaEdgeListNoAlloc(*args) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert L.galphaEdgeListNoAlloc(*args) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert int(d_n.item()) == len(want)
    np.testing.assert_array_equal(d_edges.cpu().numpy(), want)


def test_edge_list_no_alloc_bounded_wait_reports_error(engine):
    """Failure detection without a GPU fault: with the first tile made to
    withhold its count (galphaSetLimits, NULL handle) the next tile's bounded
    wait runs out, the call reports GPUDT_ERR_NOCONVERGE in *d_nEdges and
    clears the shared scratch, and the next call with the defaults restored
    is exact."""
    import torch

    L = _lib()
    L.galphaSetLimits.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    tris, want = _mesh(engine, 20000, 15, 1024)
    try:
        assert L.galphaSetLimits(None, 0, 2000, 1) == 0
        n, _ = _no_alloc(L, torch, tris, len(want))
        assert n == -5  # GPUDT_ERR_NOCONVERGE
    finally:
        assert L.galphaSetLimits(None, 0, 0, 0) == 0
    n, got = _no_alloc(L, torch, tris, len(want))
    assert n == len(want)
    np.testing.assert_array_equal(got, want)
