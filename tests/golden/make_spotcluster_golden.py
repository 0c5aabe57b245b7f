"""Makes spotcluster.npz: XPG's own clustering of strong pixels into spots (`_Accumulator`, `xpg/spotcluster.py:241-
375`: every pixel added frame by frame, one flush) on the strong pixels of seeded synthetic frames (`strong_pixels`:
Poisson background, Gaussian spots, touching pairs, and in one case a ring of signal over every frame that makes a
cluster with hundreds of peaks), classified by the oracle's restatement of XPG's classifier. Stored per case: the spot
arrays x, y, z, intensity, npix, zmin, zmax for two pixel-count ranges.

    python tests/golden/make_spotcluster_golden.py        (needs the reference checkout importable)
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

CASES = ((0, 12, 120, 140, 60, 300.0, False, False), (1, 16, 150, 160, 150, 3000.0, True, False),
         (3, 8, 200, 200, 100, 5000.0, True, True))
RANGES = ((1, 1000000), (3, 500))


def strong_pixels(seed, nf, ny, nx, nspots, bright, crowd, ring):
    """(frame, row, column, value, local background) of the strong pixels of a seeded synthetic run, frame-major."""
    from oracle import spotfind as OS
    rng = np.random.default_rng(seed)
    img = rng.poisson(0.5, (nf, ny, nx)).astype(np.float32)
    zz, yy, xx = np.mgrid[-2:3, -3:4, -3:4]
    prof = np.exp(-(zz ** 2 / 1.5 + (yy ** 2 + xx ** 2) / 2.0))
    for _ in range(nspots):
        f, y, x = rng.integers(2, nf - 2), rng.integers(4, ny - 4), rng.integers(4, nx - 4)
        amp = rng.uniform(5, bright)
        img[f - 2:f + 3, y - 3:y + 4, x - 3:x + 4] += rng.poisson(amp * prof).astype(np.float32)
        if crowd and rng.random() < 0.5:
            y2 = int(np.clip(y + rng.integers(2, 5), 4, ny - 5))
            x2 = int(np.clip(x + rng.integers(-3, 4), 4, nx - 5))
            img[f - 2:f + 3, y2 - 3:y2 + 4, x2 - 3:x2 + 4] += rng.poisson(amp * 0.7 * prof).astype(np.float32)
    if ring:
        Y, X = np.mgrid[0:ny, 0:nx]
        band = np.abs(np.hypot(Y - ny / 2, X - nx / 2) - min(ny, nx) / 3) < 2.5
        img[:, band] += rng.poisson(40.0, (nf, int(band.sum()))).astype(np.float32)
    s, m = OS.find(img, 1.0)
    k, y, x = np.nonzero(s)
    return k, y, x, img[k, y, x], m[k, y, x], ny, nx


def main():
    from refpath import import_reference
    import_reference()
    os.environ.setdefault("XPG_DEVICE", "cpu")
    import xpg.spotcluster as RC
    out = {}
    for c in CASES:
        k, y, x, v, b, ny, nx = strong_pixels(*c)
        for ri, (mn, mx) in enumerate(RANGES):
            acc = RC._Accumulator(nx, ny, mn, mx, 3.0, 2)
            for f in np.unique(k):
                sel = k == f
                acc.add(f, y[sel], x[sel], v[sel], b[sel])
            acc.flush()
            ref = acc.result()
            for kk in ("x", "y", "z", "intensity", "npix", "zmin", "zmax"):
                out[f"c{c[0]}_r{ri}_{kk}"] = getattr(ref, kk)
            print(c[0], ri, len(ref))
    np.savez_compressed(HERE / "spotcluster.npz", **out)


if __name__ == "__main__":
    main()
