"""Transfer encoding of uint32 frames: xi_pack_u8 (host code, runs here without a GPU) against its definition in
numpy, and the xi_pack_u8 -> xi_unpack_u8 round trip on the device."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from xpg_b200 import native


def _definition(src):
    plane = np.where(src < 254, src, np.where(src == 0xFFFFFFFF, 255, 254)).astype(np.uint8)
    idx = np.nonzero(plane == 254)[0]
    return plane, np.stack([idx.astype(np.uint32), src[idx]], axis=1).reshape(-1)


def _pack(src, cap, threads=0):
    lib = native.load()
    n = src.size
    plane = np.full(max(n, 1), 7, np.uint8)
    exc = np.zeros(2 * max(cap, 1), np.uint32)
    ne = C.c_int64(-1)
    rc = lib.xi_pack_u8(src.ctypes.data, n, plane.ctypes.data, exc.ctypes.data, cap, threads, C.byref(ne))
    return rc, plane[:n], exc[:2 * max(ne.value, 0)]


def _frames(n, seed, n_big):
    rng = np.random.default_rng(seed)
    src = rng.poisson(0.7, n).astype(np.uint32)
    src[rng.integers(0, n, max(n // 50, 1))] = 0xFFFFFFFF
    edge = np.array([252, 253, 254, 255, 256, 65535, 65536, 1 << 20, 0xFFFFFFFE], np.uint32)
    src[rng.integers(0, n, n_big)] = rng.choice(edge, n_big)
    return src


@pytest.mark.parametrize("n,threads", [(1, 0), (15, 1), (4097, 3), (1 << 20, 1), (3 * (1 << 20) + 5, 0),
                                       (3 * (1 << 20) + 5, 7)])
def test_pack_matches_definition(n, threads):
    src = _frames(n, n, max(n // 300, 3))
    plane, exc = _definition(src)
    rc, p, e = _pack(src, n, threads)
    assert rc == native.XI_OK
    assert np.array_equal(p, plane)
    assert np.array_equal(e, exc)


def test_pack_empty_and_arguments():
    lib = native.load()
    ne = C.c_int64(5)
    assert lib.xi_pack_u8(None, 0, None, None, 0, 0, C.byref(ne)) == native.XI_OK and ne.value == 0
    src = np.zeros(16, np.uint32)
    plane = np.zeros(16, np.uint8)
    assert lib.xi_pack_u8(src.ctypes.data, -1, plane.ctypes.data, None, 0, 0, C.byref(ne)) == native.XI_E_ARG
    assert lib.xi_pack_u8(src.ctypes.data, 16, plane.ctypes.data, None, 0, 0, None) == native.XI_E_ARG
    assert lib.xi_pack_u8(src.ctypes.data, 1 << 33, plane.ctypes.data, None, 0, 0, C.byref(ne)) == native.XI_E_LIMIT


def test_pack_exception_list_full():
    src = _frames(50000, 3, 500)
    _, exc = _definition(src)
    k = exc.size // 2
    rc, _, e = _pack(src, k, 2)
    assert rc == native.XI_OK and e.size == 2 * k
    rc, _, _ = _pack(src, k - 1, 2)
    assert rc == native.XI_E_LIMIT
    assert b"exc_cap" in native.load().xi_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 16, 17, 65536 + 3, 5 * 16384 + 1, 2 * 4148 * 4362])
def test_unpack_round_trip(n):
    import torch
    lib = native.load()
    src = _frames(n, n + 1, max(n // 1000, 2))
    plane, exc = _definition(src)
    d_plane = torch.from_numpy(plane).cuda()
    d_exc = torch.from_numpy(exc.view(np.int32)).cuda() if exc.size else None
    out = torch.full((n,), 12345, dtype=torch.int32, device="cuda")
    rc = lib.xi_unpack_u8(native.ptr(d_plane), n, native.ptr(d_exc), exc.size // 2, native.ptr(out),
                          native.stream_handle())
    native.check(rc, "xi_unpack_u8")
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), src)


@pytest.mark.gpu
@pytest.mark.parametrize("n,off", [(1, 0), (15, 1), (16, 0), (4099, 3), (1 << 20, 0), (3 * (1 << 20) + 7, 5)])
def test_upload_round_trip(n, off):
    """xi_upload copies from page-locked host memory at any offset and length, bit for bit."""
    import torch
    lib = native.load()
    host = torch.randint(0, 256, (n + off,), dtype=torch.uint8).pin_memory()
    out = torch.zeros(n + 16, dtype=torch.uint8, device="cuda")
    rc = lib.xi_upload(C.c_void_p(host.data_ptr() + off), C.c_void_p(out.data_ptr() + (off & 1)), n,
                       native.stream_handle())
    native.check(rc, "xi_upload")
    torch.cuda.synchronize()
    assert torch.equal(out[(off & 1):(off & 1) + n].cpu(), host[off:off + n])


@pytest.mark.gpu
def test_upload_rejects_pageable_memory():
    import torch
    lib = native.load()
    src = np.arange(64, dtype=np.uint8)                     # pageable: refused before any launch
    out = torch.zeros(64, dtype=torch.uint8, device="cuda")
    assert lib.xi_upload(src.ctypes.data, native.ptr(out), 64, native.stream_handle()) == native.XI_E_ARG


@pytest.mark.gpu
def test_h2d_ring_wraps():
    """The upload ring gives every upload its own bytes while regions are reused (more than the ring's size in
    flight across a run of uploads)."""
    import torch
    from xpg_b200 import device as D
    rng = np.random.default_rng(5)
    arrays = [rng.integers(0, 1 << 30, size=int(rng.integers(1, 3 << 20)), dtype=np.int64) for _ in range(40)]
    outs = [D.h2d(a) for a in arrays]
    torch.cuda.synchronize()
    for a, o in zip(arrays, outs):
        assert np.array_equal(o.cpu().numpy(), a)
