"""Oracle of the strong-pixel classifier of spot finding: TEST INFRASTRUCTURE (see oracle/__init__.py).

Reference: `xpg/spotfind.py:27-97` (`_box_sum`, `_dilate`, `_dispersion`, `make_finder`): the dispersion test
(Kabsch 2010) on a (2 nby + 1) x (2 nbx + 1) window, then the extended pass that re-estimates the local background
in a window twice as wide from pixels away from first-pass signal. float32 throughout, one operation at a time in the
reference's order; window sums run along x then along y, each over its window in increasing coordinate (zero
outside the frame), the order the reference's pooling sums in (pinned by tests/golden/spotfind.npz, made by running
XPG's own classifier).
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
DISPERSION_SIGMA_B = 6.0


def box_sum(a, hy, hx):
    """(B, ny, nx) float32 window sums, zero padded: along x first, then along y, each in increasing offset."""
    a = np.asarray(a, F32)
    B, ny, nx = a.shape
    p = np.zeros((B, ny, nx + 2 * hx), F32)
    p[:, :, hx:hx + nx] = a
    h = np.zeros((B, ny, nx), F32)
    for d in range(2 * hx + 1):
        h = h + p[:, :, d:d + nx]
    q = np.zeros((B, ny + 2 * hy, nx), F32)
    q[:, hy:hy + ny] = h
    v = np.zeros((B, ny, nx), F32)
    for d in range(2 * hy + 1):
        v = v + q[:, d:d + ny]
    return v


def dilate(m, r):
    return box_sum(m.astype(F32), r, r) > 0


def dispersion(img, valid, gain, hy, hx, n_b, n_s, min_local):
    g = F32(gain)
    w = valid.astype(F32)
    x = np.where(valid, img, F32(0.0)).astype(F32)
    n = box_sum(w, hy, hx)
    s1 = box_sum(x, hy, hx)
    s2 = box_sum(x * x, hy, hx)
    nn = np.maximum(n, F32(2.0))
    mean = s1 / nn
    var = np.maximum((s2 - s1 * mean) / (nn - F32(1.0)), F32(0.0))
    disp_thr = g * (F32(1.0) + F32(n_b) * np.sqrt(F32(2.0) / (nn - F32(1.0))))
    disp = var > disp_thr * np.maximum(mean, F32(1e-6))
    strong = (x - mean) > F32(n_s) * np.sqrt(g * np.maximum(mean, F32(1.0)))
    ok = valid & (n >= F32(min_local))
    return ok & disp & strong, mean


def find(img, gain, nbx=3, nby=3, signal_pixel=3.0, background_pixel=2.0, min_local=2, extended=True):
    """(strong, mean) of frames img (B, ny, nx) float32 (negative: not valid)."""
    img = np.asarray(img, F32)
    g = F32(gain)
    hx, hy = int(nbx), int(nby)
    valid = img >= 0
    s1, mean1 = dispersion(img, valid, gain, hy, hx, DISPERSION_SIGMA_B, signal_pixel, min_local)
    if not extended:
        return s1, mean1
    sig1 = np.sqrt(g * np.maximum(mean1, F32(0.5)))
    bgpix = valid & ~dilate(s1, 1) & (img <= mean1 + F32(background_pixel) * sig1)
    w = bgpix.astype(F32)
    x = np.where(bgpix, img, F32(0.0)).astype(F32)
    hy2, hx2 = 2 * hy + 1, 2 * hx + 1
    n = box_sum(w, hy2, hx2)
    m1 = box_sum(x, hy2, hx2)
    m2 = box_sum(x * x, hy2, hx2)
    nn = np.maximum(n, F32(2.0))
    mean = m1 / nn
    var = np.maximum((m2 - m1 * mean) / (nn - F32(1.0)), F32(0.0))
    sig = np.sqrt(np.maximum(g * np.maximum(mean, F32(0.5)), var))
    strong = valid & (n >= F32(4 * min_local)) & ((img - mean) > F32(signal_pixel) * sig)
    return strong & dilate(s1, 2), mean
