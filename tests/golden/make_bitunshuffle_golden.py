"""Makes bitunshuffle.npz: LZ4-stage outputs (bit-shuffled bytes, as a bitshuffle-LZ4 chunk's blocks decompress)
and the frames XPG's own device decoder gives for them (`unshuffle_frame_torch`, `xpg/io/bslz4.py:85-121`, run on
CPU tensors here), plus XPG's numpy `_bitunshuffle` (`:28-32`) of one shuffled group. This pins the bit order of the
oracle's and the library's unshuffle (and the oracle's test encoder, their inverse) to the reference's.

Cases: uint32 and uint16 elements; frames of several sizes around the 8192-byte block (a partial last block, n % 8
trailing elements stored as they are); counts below 2^24 (exact in XPG's float32 output) with flagged all-ones pixels.

    XPG_REFERENCE_ROOT=<reference checkout> python tests/golden/make_bitunshuffle_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import bslz4 as OB  # noqa: E402

# (XPG's torch unshuffle cannot take a shuffled run of exactly 8 elements, a one-byte bit plane: no case has one)
CASES = [(4, 64), (4, 37 * 61), (4, 3 * 2048 + 29), (4, 2048 * 5), (2, 4096 + 7), (2, 3 * 4096 + 40), (2, 501)]


def frame(esize, n, seed):
    rng = np.random.default_rng(seed)
    if esize == 4:
        v = rng.integers(0, 1 << 24, n, dtype=np.int64).astype(np.uint32)
        v[rng.random(n) < 0.05] = 0xFFFFFFFF
    else:
        v = rng.integers(0, 0xFFFF, n, dtype=np.int64).astype(np.uint16)
        v[rng.random(n) < 0.05] = 0xFFFF
    return v


def staged(v, esize):
    """LZ4-stage output of v with 8192-byte blocks (the oracle's test encoder, block by block)."""
    raw = v.view(np.uint8)
    n = v.size
    belem = 8192 // esize
    parts, done = [], 0
    while done < n:
        m = min(belem, n - done)
        m8 = m - m % 8
        if m8:
            parts.append(OB.bitshuffle(raw[done * esize:(done + m8) * esize], m8, esize))
        parts.append(raw[(done + m8) * esize:(done + m) * esize])
        done += m
    return np.concatenate(parts), belem


if __name__ == "__main__":
    import torch
    from refpath import import_reference
    import_reference()
    from xpg.io import bslz4 as RB
    save = {}
    for i, (esize, n) in enumerate(CASES):
        v = frame(esize, n, 100 + i)
        st, belem = staged(v, esize)
        img = RB.unshuffle_frame_torch(torch.from_numpy(st.copy()), n, esize, belem).numpy()
        flagged = v == (0xFFFFFFFF if esize == 4 else 0xFFFF)
        assert np.array_equal(img[~flagged], v[~flagged].astype(np.float32)) and (img[flagged] == -1.0).all()
        save[f"c{i}_esize"] = np.int64(esize)
        save[f"c{i}_n"] = np.int64(n)
        save[f"c{i}_block"] = np.int64(belem)
        save[f"c{i}_staged"] = st
        save[f"c{i}_xpg_frame"] = img
    # XPG's numpy unshuffle of one 64-element group of 4-byte elements
    grp = np.random.default_rng(7).integers(0, 256, 64 * 4, dtype=np.int64).astype(np.uint8)
    save["np_in"] = grp
    save["np_out"] = RB._bitunshuffle(grp, 64, 4)
    np.savez_compressed(HERE / "bitunshuffle.npz", **save)
    print((HERE / "bitunshuffle.npz").stat().st_size)
