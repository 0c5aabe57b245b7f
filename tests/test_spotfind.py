"""Strong-pixel classifier of spot finding (`xpg/spotfind.py:27-97`): the oracle against XPG's own classifier's
results (tests/golden/spotfind.npz, made by tests/golden/make_spotfind_golden.py), and on the GPU the library's
kernels against the oracle, bit for bit (masks and local means), on frames with masked pixels, a masked band and spots
bright enough that float32 window sums of squares round."""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import spotfind as OS

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
import make_spotfind_golden as M  # noqa: E402


@pytest.fixture(scope="module")
def gold():
    z = np.load(HERE / "golden" / "spotfind.npz")
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("trial", range(6))
def test_oracle_matches_reference(trial, gold):
    img = M.frames(trial)
    for si, st in enumerate(M.SETTINGS):
        s, m = OS.find(img, float(gold[f"t{trial}_s{si}_gain"]), **st)
        assert np.array_equal(np.packbits(s.reshape(-1)), gold[f"t{trial}_s{si}_strong"]), (trial, si)
        assert hashlib.sha256(m.astype(np.float32).tobytes()).hexdigest() == str(gold[f"t{trial}_s{si}_mean_sha"])


@pytest.mark.gpu
@pytest.mark.parametrize("trial", range(6))
def test_device_classifier_matches_oracle(trial, gold):
    import torch
    from xpg_b200.spotfind import make_finder
    img = M.frames(trial)
    for si, st in enumerate(M.SETTINGS):
        gain = float(gold[f"t{trial}_s{si}_gain"])
        s_ref, m_ref = OS.find(img, gain, **st)
        s, m = make_finder(**st)(torch.from_numpy(img).cuda(), gain)
        assert np.array_equal(s.cpu().numpy(), s_ref), (trial, si, int(s.sum()), int(s_ref.sum()))
        assert np.array_equal(m.cpu().numpy(), m_ref), (trial, si)
    one, _ = make_finder()(torch.from_numpy(img[0]).cuda(), 1.0)        # a single (ny, nx) frame
    assert one.shape == img.shape[1:]


@pytest.mark.gpu
def test_device_classifier_full_frame():
    """A 4148 x 4362 frame (config-2 detector): the same as the oracle, both passes."""
    import torch
    from xpg_b200.spotfind import make_finder
    rng = np.random.default_rng(3)
    img = rng.poisson(0.2, (1, 4362, 4148)).astype(np.float32)
    img[0, :, ::259] = -1.0
    ys, xs = rng.integers(5, 4357, 3000), rng.integers(5, 4143, 3000)
    for y, x in zip(ys, xs):
        img[0, y - 1:y + 2, x - 1:x + 2] += rng.integers(5, 200)
    s_ref, m_ref = OS.find(img, 1.0)
    s, m = make_finder()(torch.from_numpy(img).cuda(), 1.0)
    assert np.array_equal(s.cpu().numpy(), s_ref)
    assert np.array_equal(m.cpu().numpy(), m_ref)
