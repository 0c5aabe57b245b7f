"""Makes findspots.npz: XPG's own `find_spots` (`xpg/spotfind.py:122-300`, on the CPU: the classifier in torch
eagerly, the clustering in this process) on an in-memory image set of seeded uint32 frames (`raw_frames`: Poisson
background, Gaussian spots with touching pairs, flagged pixels, counts over the overload threshold), frames 1-14 and
16-23 (a gap), batches of 4 frames, a static mask: the spot arrays in XPG's order.

    python tests/golden/make_findspots_golden.py        (needs the reference checkout importable)
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
NY, NX, NF, OVERLOAD = 150, 170, 23, 1 << 20
FRAMES = list(range(1, 15)) + list(range(16, 24))
KW = dict(gain=1.0, min_pixels=3, max_pixels=2000, batch=4)


def raw_frames():
    rng = np.random.default_rng(21)
    img = rng.poisson(0.6, (NF, NY, NX)).astype(np.uint32)
    zz, yy, xx = np.mgrid[-2:3, -3:4, -3:4]
    prof = np.exp(-(zz ** 2 / 1.5 + (yy ** 2 + xx ** 2) / 2.0))
    for _ in range(120):
        f, y, x = rng.integers(2, NF - 2), rng.integers(4, NY - 4), rng.integers(4, NX - 4)
        amp = rng.uniform(5, 3000)
        img[f - 2:f + 3, y - 3:y + 4, x - 3:x + 4] += rng.poisson(amp * prof).astype(np.uint32)
        if rng.random() < 0.4:
            y2, x2 = int(np.clip(y + rng.integers(2, 5), 4, NY - 5)), int(np.clip(x + rng.integers(-3, 4), 4, NX - 5))
            img[f - 2:f + 3, y2 - 3:y2 + 4, x2 - 3:x2 + 4] += rng.poisson(amp * 0.7 * prof).astype(np.uint32)
    img[rng.random(img.shape) < 0.003] = 0xFFFFFFFF
    img[3, 50, 60] = OVERLOAD + 5
    return img


def static_mask():
    m = np.ones((NY, NX), bool)
    m[:, 100:103] = False
    return m


def main():
    from refpath import import_reference
    import_reference()
    for k, v in (("XPG_DEVICE", "cpu"), ("XPG_COMPILE", "0"), ("XPG_SPOTS_PROCESS", "0"), ("XPG_DECODE_PROCS", "0")):
        os.environ.setdefault(k, v)
    from xpg.io.images import ImageSet
    from xpg.spotfind import find_spots
    raw = raw_frames()

    class MemImages(ImageSet):
        def __init__(self):
            super().__init__(min_valid=0.0, overload=OVERLOAD)
            self.nx, self.ny, self.first, self.last = NX, NY, 1, NF

        def _read_native(self, frame):
            r = raw[frame - 1]
            return r, r == np.iinfo(r.dtype).max

    spots = find_spots(MemImages(), FRAMES, mask=static_mask(), verbose=False, **KW)
    out = {k: getattr(spots, k) for k in ("x", "y", "z", "intensity", "npix", "zmin", "zmax")}
    np.savez_compressed(HERE / "findspots.npz", **out)
    print(len(spots))


if __name__ == "__main__":
    main()
