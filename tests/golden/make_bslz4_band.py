"""Makes bslz4_band.bin: the bitshuffle-LZ4 chunk (HDF5 filter 32008 layout, 8192-byte blocks) of a 256 x 4148 uint32
band of a config-2 frame (Poisson background 0.2, seed 11, flagged module-gap columns every 259 pixels), encoded by
the oracle's test encoder. bench.py --decode regenerates the band with the same seed, decodes the chunk with the
library and checks it against the band before timing.

    python tests/golden/make_bslz4_band.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import bslz4 as OB  # noqa: E402

NY, NX, SEED = 256, 4148, 11


def band():
    rng = np.random.default_rng(SEED)
    b = rng.poisson(0.2, (NY, NX)).astype(np.uint32)
    b[:, ::259] = 0xFFFFFFFF
    return b


if __name__ == "__main__":
    (HERE / "bslz4_band.bin").write_bytes(OB.encode_chunk(band(), 4))
    print((HERE / "bslz4_band.bin").stat().st_size)
