"""The allocation-free neighbour search, `xi_knn_noalloc`, called through the C ABI.

It exists for callers that cannot allocate device memory: a program that binds libxpgi.so through a plain C FFI
next to a framework that has already taken the GPU's memory into its own pool. It keeps its scratch memory in an
array inside the library, so these checks compare it with `xi_knn` (the same search on a caller-provided workspace):
two calls in a row, the second smaller and with fewer columns, so that counters left over from the first call would
show, then a call whose bounds need more grid cells than the array holds (the no-alloc form takes coarser cells
there), and a call above the array's point limit, which must fail cleanly. Neighbour indices and distances are
integer / exact results: they must be identical.

The file name keeps it last in collection order; it passes alone in a fresh process as well as after the suite.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from xpg_b200 import native as N

pytestmark = pytest.mark.gpu


def _query(n, k, extent, seed, scales=(7.5, 1.25)):
    rng = np.random.default_rng(seed)
    pts = {a: torch.as_tensor(rng.uniform(0.0, e, n)).cuda() for a, e in zip("xyz", extent)}
    q = N.XiKnn()
    q.n, q.k, q.radius = n, k, 12.0
    q.x, q.y, q.z = N.ptr(pts["x"]), N.ptr(pts["y"]), N.ptr(pts["z"])
    q.sx, q.sz = scales
    q.lo[:] = [0.0, 0.0, 0.0]
    q.hi[:] = [extent[0] / scales[0], extent[1] / scales[0], extent[2] / scales[1]]
    return q, pts


def _outputs(n, k):
    return (torch.full((n, k), -7, dtype=torch.int32, device="cuda"),
            torch.full((n, k), -7.0, dtype=torch.float64, device="cuda"))


def _with_workspace(lib, q):
    ws = torch.empty(int(lib.xi_knn_workspace(C.byref(q))), dtype=torch.uint8, device="cuda")
    j, d = _outputs(q.n, q.k)
    N.check(lib.xi_knn(C.byref(q), N.ptr(ws), ws.numel(), N.ptr(j), N.ptr(d), N.stream_handle()), "xi_knn")
    return j.cpu().numpy(), d.cpu().numpy()


def _without_allocation(lib, q):
    j, d = _outputs(q.n, q.k)
    N.check(lib.xi_knn_noalloc(C.byref(q), N.ptr(j), N.ptr(d), N.stream_handle()), "xi_knn_noalloc")
    torch.cuda.synchronize()
    return j.cpu().numpy(), d.cpu().numpy()


def test_noalloc_knn_matches_workspace_form_on_consecutive_calls():
    lib = N.load()
    cases = [(60_000, 8, (9000.0, 7000.0, 100.0), 11),      # ~5 neighbours in reach: full and partial lists
             (20_000, 5, (3000.0, 2500.0, 60.0), 12),       # a smaller second call on the same array
             (300_000, 8, (40000.0, 40000.0, 100.0), 14)]  # ~1.4M cells of the search radius: coarser cells here
    for n, k, extent, seed in cases:
        q, keep = _query(n, k, extent, seed)
        j_ref, d_ref = _with_workspace(lib, q)
        j, d = _without_allocation(lib, q)
        assert np.isfinite(d_ref).any() and (~np.isfinite(d_ref)).any()
        np.testing.assert_array_equal(j, j_ref)
        np.testing.assert_array_equal(d, d_ref)


def test_noalloc_knn_rejects_more_points_than_its_array():
    lib = N.load()
    q, keep = _query(1024, 8, (900.0, 700.0, 10.0), 13)
    q.n = N.XI_KNN_NOALLOC_MAX_POINTS + 1          # refused on the host before any launch
    j, d = _outputs(1024, 8)
    rc = lib.xi_knn_noalloc(C.byref(q), N.ptr(j), N.ptr(d), N.stream_handle())
    assert rc == N.XI_E_LIMIT
    assert "XI_KNN_NOALLOC_MAX_POINTS" in lib.xi_last_error().decode()
    assert (j.cpu().numpy() == -7).all()
