"""CPU restatement of the forward-model likelihood passes (TEST INFRASTRUCTURE: the checker of the library's
xi_fm_scatter / xi_fm_gather, never product code).

XPG's pixel-level forward model (xpg/forward/) keeps, per chunk of reflections, separable profile factors: a
reflection's fraction in voxel (z, y, x) of its box is f = sum_t R[t, row, z] * P[t, row, y, x] (the product of a
rocking-curve factor and a detector-profile factor per term; `expand_terms`, xpg/forward/model.py:197-203). The
voxels of a window of frames [f0, f1) x rows [y0, y0 + ny) x columns [x0, x0 + nx) are indexed densely,
(kz * ny + ky) * nx + kx with kz = iz0 + z - f0, ky = iy0 + y - y0, kx = ix0 + x - x0; voxels outside the window are
dropped (`WindowModel.vid`, :381-392). The passes (`WindowModel.mu`, `grad_ratio`, `grad_newton`, :476-577; fused
on CUDA by the Triton kernels of xpg/forward/kernels.py:34-103):

    scatter:       mu[v] += I_row * f + beta_row                 over every in-window voxel of each box
    grad_ratio:    g[row] += sum f * A[v] / M[v]                 over in-window voxels with NS[v] >= 0
    grad_newton:   g[row] += sum f * (1 - max(NS[v], 0) / M[v]), fd[row] += sum f^2 / max(M[v], 1e-6)   (same voxels)

f and every product are float32 as XPG computes them (separate roundings, no fused multiply-add); the sums are
accumulated in float64 here (XPG's and the device's float32 sums differ from them by float32 rounding in another
order, which the tests' tolerance covers). Pinned on XPG's own passes run on the same inputs
(tests/golden/forward.npz, made by tests/golden/make_forward_golden.py).
"""
from __future__ import annotations

import numpy as np


def fractions(R, P):
    """f (n, Dz, b, b) float32 = sum_t R[t][:, :, None, None] * P[t][:, None] (products rounded, then summed)."""
    f = None
    for t in range(R.shape[0]):
        g = (R[t][:, :, None, None] * P[t][:, None]).astype(np.float32)
        f = g if f is None else (f + g).astype(np.float32)
    return f


def voxel_index(iz0, iy0, ix0, Dz, b, win):
    """Dense window index (n, Dz, b, b) of every box voxel, -1 outside the window."""
    f0, f1, y0, ny, x0, nx = (int(v) for v in win)
    kz = np.asarray(iz0, np.int64)[:, None] + np.arange(Dz)[None] - f0
    ky = np.asarray(iy0, np.int64)[:, None] + np.arange(b)[None] - y0
    kx = np.asarray(ix0, np.int64)[:, None] + np.arange(b)[None] - x0
    ok = ((kz >= 0) & (kz < f1 - f0))[:, :, None, None] & ((ky >= 0) & (ky < ny))[:, None, :, None] \
        & ((kx >= 0) & (kx < nx))[:, None, None, :]
    lin = (kz[:, :, None, None] * ny + ky[:, None, :, None]) * nx + kx[:, None, None, :]
    return np.where(ok, lin, -1)


def scatter(mu, groups, I, beta, win):
    """mu (float64 copy of the window's starting values) += I f + beta over each group's in-window voxels. groups:
    dicts of R (T, n, Dz), P (T, n, b, b), iz0, iy0, ix0, rows."""
    out = np.asarray(mu, np.float64).copy()
    for g in groups:
        R, P = g["R"], g["P"]
        f = fractions(R, P)
        v = voxel_index(g["iz0"], g["iy0"], g["ix0"], R.shape[2], P.shape[-1], win)
        val = (f * I[g["rows"]][:, None, None, None]).astype(np.float32)
        if beta is not None and len(beta):
            val = (val + beta[g["rows"]][:, None, None, None]).astype(np.float32)
        ok = v >= 0
        np.add.at(out, v[ok], val[ok].astype(np.float64))
    return out


def gather(groups, win, n, A, M, NS, mode):
    """mode 0: g[row] = sum f A / M; mode 1: g[row] = sum f (1 - max(NS, 0) / M), fd[row] = sum f^2 / max(M, 1e-6);
    over each box's in-window voxels with NS >= 0. Returns (g, fd) float64 (fd None for mode 0)."""
    g_out = np.zeros(n, np.float64)
    fd_out = np.zeros(n, np.float64) if mode == 1 else None
    for g in groups:
        R, P = g["R"], g["P"]
        f = fractions(R, P)
        v = voxel_index(g["iz0"], g["iy0"], g["ix0"], R.shape[2], P.shape[-1], win)
        vc = np.maximum(v, 0)
        ns = np.asarray(NS)[vc].astype(np.float32)
        use = (v >= 0) & (ns >= 0)
        m = np.asarray(M, np.float32)[vc]
        if mode == 0:
            w = (np.asarray(A, np.float32)[vc] / m).astype(np.float32)
        else:
            w = (np.float32(1.0) - (np.maximum(ns, np.float32(0.0)) / m).astype(np.float32)).astype(np.float32)
            d = ((f * f).astype(np.float32) / np.maximum(m, np.float32(1e-6))).astype(np.float32)
            np.add.at(fd_out, g["rows"], np.where(use, d, 0.0).astype(np.float64).sum(axis=(1, 2, 3)))
        t = (f * w).astype(np.float32)
        np.add.at(g_out, g["rows"], np.where(use, t, 0.0).astype(np.float64).sum(axis=(1, 2, 3)))
    return g_out, fd_out
