"""Oracle of the frame preparation and shoebox gather: TEST INFRASTRUCTURE (see oracle/__init__.py).

References: pixel encoding `xpg/io/images.py:72-102` (Eiger flags `:408-419`), mask ceiling and super-pixel sums
`xpg/integrate.py:667-699`, gather into shoebox slots `xpg/integrate.py:704-787`, binned-bin decoding
`xpg/shoebox.py:264-268` and the incomplete-bin rule `xpg/integrate.py:483-488`.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
SB_OFF = F32(3.0)


def prepare_frame(raw, overload, min_valid=0, mask=None):
    """float32 frame: counts, -2 overloaded, -1 flagged / below min_valid, masked pixels min(value, -1)."""
    raw = np.asarray(raw)
    img = raw.astype(F32)
    bad = raw == np.iinfo(raw.dtype).max
    if min_valid > 0:
        bad |= raw < min_valid
    if overload is not None:
        img[raw >= overload] = F32(-2.0)
    img[bad] = F32(-1.0)
    if mask is not None:
        m = ~np.asarray(mask, bool)
        img[m] = np.minimum(img[m], F32(-1.0))
    return img


def superpixel_frame(prep, s):
    """s x s sums (row-major order of the s^2 terms, float32); a super-pixel holding a negative pixel is -2 when its
    smallest value is <= -1.5, else -1. Incomplete super-pixels at the far edges are left out."""
    ny, nx = prep.shape[0] // s, prep.shape[1] // s
    a = prep[:ny * s, :nx * s]
    dst = a[0::s, 0::s].copy()
    mn = dst.copy()
    for i in range(s):
        for j in range(s):
            if i or j:
                v = a[i::s, j::s]
                dst = (dst + v).astype(F32)
                mn = np.minimum(mn, v)
    neg = mn < 0
    dst[neg] = np.where(mn[neg] <= -1.5, F32(-2.0), F32(-1.0))
    return dst


def window(img, iy0, ix0, bx):
    """bx x bx window with top-left (iy0, ix0) in array indices; outside the image -1."""
    out = np.full((bx, bx), F32(-1.0))
    ny, nx = img.shape
    y0, y1 = max(iy0, 0), min(iy0 + bx, ny)
    x0, x1 = max(ix0, 0), min(ix0 + bx, nx)
    if y1 > y0 and x1 > x0:
        out[y0 - iy0:y1 - iy0, x0 - ix0:x1 - ix0] = img[y0:y1, x0:x1]
    return out


def gather_shoebox(prepared, frame_ids, iz0, fb, Dz, bx, iy0, ix0):
    """Shoebox (Dz, bx, bx) of one reflection from `prepared[fi]` (the frame of 0-based index fi, already at the
    reflection's super-pixel scale) over the frames `frame_ids` that were read, in order. Unrecorded slots -3."""
    if fb == 1:
        arr = np.zeros((Dz, bx, bx), F32)
        for fi in frame_ids:
            k = fi - iz0
            if 0 <= k < Dz:
                arr[k] = window(prepared[fi], iy0, ix0, bx) + SB_OFF
        return (arr - SB_OFF).astype(F32)
    acc = np.zeros((Dz, bx, bx), F32)
    cnt = np.zeros(Dz, np.int64)
    for fi in frame_ids:
        k = fi - iz0
        if 0 <= k < Dz * fb:
            k //= fb
            v = window(prepared[fi], iy0, ix0, bx)
            neg = v < 0
            v[neg] = np.where(v[neg] == -2.0, F32(np.nan), F32(np.inf))
            acc[k] = (acc[k] + v).astype(F32)
            cnt[k] += 1
    return (decode_bins(acc, cnt, fb) - SB_OFF).astype(F32)


def decode_bins(acc, cnt, fb):
    """Stored (value + 3) form of binned sums (`xpg/shoebox.py:264-268` and `xpg/integrate.py:483-488`): an
    overloaded frame (NaN) makes the bin -2, a masked one (+inf) -1 (overload wins), bins holding fewer than fb
    frames are unrecorded (0). acc: (Dz, ...) IEEE-encoded sums; cnt: (Dz,) frames per bin."""
    arr = np.nan_to_num(np.asarray(acc, F32), nan=-2.0, posinf=-1.0, neginf=-1.0).astype(F32) + SB_OFF
    arr[np.asarray(cnt) < fb] = F32(0.0)
    return arr
