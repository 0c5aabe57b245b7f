"""Forward-model likelihood passes on the device: a drop-in for XPG's `xpg.forward.kernels` (the fused Triton
scatter / gather of the window model, xpg/forward/kernels.py:28-134), with the same functions and arguments, computed
by the library's sm_100a kernels (xi_fm_scatter, xi_fm_gather).

    scatter(mu, R, P, I, beta, iz0, iy0, ix0, win)                mu[v] += I f + beta over the in-window voxels
    gather(g, fd, R, P, rows, iz0, iy0, ix0, win, A, M, NS, mode)  mode 0: g[rows] += sum f A / M;
                                                                   mode 1: g[rows] += sum f (1 - NS / M),
                                                                           fd[rows] += sum f^2 / M   (NS >= 0)

R: (T, n, Dz), P: (T, n, b, b) float32 contiguous CUDA tensors (T = 1, or 2 with the halo); iz0 / iy0 / ix0 int64
(n); win: an object with f0, f1, y0, ny, x0, nx (XPG's `Window`). Installing it in place of XPG's module
(`sys.modules["xpg.forward.kernels"] = xpg_b200.forward`) routes XPG's forward integrator through these kernels.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import native as N

_NS = {torch.int16: N.XI_FM_NS_I16, torch.int32: N.XI_FM_NS_I32, torch.float32: N.XI_FM_NS_F32}


def available(dev) -> bool:
    """The device passes run on CUDA devices (the library is required; there is no CPU path here)."""
    return getattr(dev, "type", str(dev)) == "cuda"


def _boxes(R, P, iz0, iy0, ix0):
    for name, t, dt in (("R", R, torch.float32), ("P", P, torch.float32), ("iz0", iz0, torch.int64),
                        ("iy0", iy0, torch.int64), ("ix0", ix0, torch.int64)):
        if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
            raise TypeError(f"{name}: a contiguous {dt} CUDA tensor")
    T, n, Dz = R.shape
    b = P.shape[-1]
    if tuple(P.shape) != (T, n, b, b) or any(t.numel() != n for t in (iz0, iy0, ix0)):
        raise ValueError("R (T, n, Dz), P (T, n, b, b) and origins (n) disagree")
    s = N.XiFmBoxes()
    s.n, s.n_terms, s.Dz, s.b = int(n), int(T), int(Dz), int(b)
    s.R, s.P, s.iz0, s.iy0, s.ix0 = (N.ptr(t) for t in (R, P, iz0, iy0, ix0))
    return s


def _window(win):
    w = N.XiFmWindow()
    w.f0, w.nf = int(win.f0), int(win.f1 - win.f0)
    w.y0, w.ny, w.x0, w.nx = int(win.y0), int(win.ny), int(win.x0), int(win.nx)
    return w


def _check(rc, what):
    if rc != N.XI_OK:
        raise RuntimeError(f"{what}: " + N.load().xi_fm_last_error().decode())


def scatter(mu, R, P, I, beta, iz0, iy0, ix0, win):
    """mu[voxel] += I_row f + beta_row over the in-window voxels of each reflection's box (WindowModel.mu)."""
    if R.shape[1] == 0:
        return mu
    N.require_cuda()
    b = _boxes(R, P, iz0, iy0, ix0)
    w = _window(win)
    _check(N.load().xi_fm_scatter(C.byref(b), C.byref(w), N.ptr(I), N.ptr(beta) if beta is not None else None,
                                  N.ptr(mu), N.stream_handle()), "xi_fm_scatter")
    return mu


def gather(g, fd, R, P, rows, iz0, iy0, ix0, win, A, M, NS, mode):
    """mode 0: g[rows] += sum f A / M; mode 1: g[rows] += sum f (1 - NS / M), fd[rows] += sum f^2 / M (voxels with
    NS >= 0, inside the window)."""
    if R.shape[1] == 0:
        return g, fd
    N.require_cuda()
    if NS.dtype not in _NS:
        raise TypeError("NS: int16, int32 or float32")
    b = _boxes(R, P, iz0, iy0, ix0)
    w = _window(win)
    rows = rows.to(torch.int64).contiguous() if rows is not None else None
    _check(N.load().xi_fm_gather(C.byref(b), C.byref(w), N.ptr(rows) if rows is not None else None,
                                 N.ptr(A) if A is not None else None, N.ptr(M), N.ptr(NS), _NS[NS.dtype], int(mode),
                                 N.ptr(g), N.ptr(fd) if fd is not None else None, N.stream_handle()),
           "xi_fm_gather")
    return g, fd
