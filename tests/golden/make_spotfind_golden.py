"""Makes spotfind.npz: XPG's own strong-pixel classifier (`make_finder`, `xpg/spotfind.py:57-97`, torch on the CPU)
run on seeded synthetic frames (`frames()`: Poisson backgrounds from 0.05 to 30 counts, Gaussian spots up to 60000
counts whose squared sums exceed float32's exact integers, masked -1 / -2 pixels and a masked column band), for the
settings in SETTINGS: the strong masks (packed bits) and the sha256 of the local means' float32 bytes.

    python tests/golden/make_spotfind_golden.py        (needs the reference checkout importable)
"""
from __future__ import annotations

import hashlib
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SETTINGS = (dict(), dict(extended=False), dict(nbx=2, nby=4, min_local=3, signal_pixel=2.5, background_pixel=1.5))
GAINS = (1.0, 1.3, 0.8)


def frames(trial):
    rng = np.random.default_rng(100 + trial)
    B, ny, nx = 2, 97 + trial * 13, 131 + trial * 7
    img = rng.poisson([0.3, 2.0, 8.0, 0.05, 30.0, 1.0][trial], (B, ny, nx)).astype(np.float32)
    yy, xx = np.mgrid[-3:4, -3:4]
    for _ in range(20):
        b, y, x = rng.integers(0, B), rng.integers(3, ny - 3), rng.integers(3, nx - 3)
        amp = [20, 500, 20000, 60000][rng.integers(0, 4)]
        img[b, y - 3:y + 4, x - 3:x + 4] += np.round(amp * np.exp(-(yy ** 2 + xx ** 2) / 2.0)).astype(np.float32)
    img[rng.random(img.shape) < 0.02] = -1.0
    img[rng.random(img.shape) < 0.002] = -2.0
    img[:, :, 40:42] = -1.0
    return img


def main():
    from refpath import import_reference
    import_reference()
    os.environ.setdefault("XPG_DEVICE", "cpu")
    import torch
    import xpg.spotfind as SF
    out = {}
    for trial in range(6):
        img = frames(trial)
        for si, st in enumerate(SETTINGS):
            gain = GAINS[(trial + si) % len(GAINS)]
            s, m = SF.make_finder(**st)(torch.from_numpy(img), gain)
            out[f"t{trial}_s{si}_strong"] = np.packbits(s.numpy().reshape(-1))
            out[f"t{trial}_s{si}_mean_sha"] = np.array(hashlib.sha256(m.numpy().tobytes()).hexdigest())
            out[f"t{trial}_s{si}_gain"] = np.float64(gain)
            print(trial, si, int(s.sum()))
    np.savez_compressed(HERE / "spotfind.npz", **out)


if __name__ == "__main__":
    main()
