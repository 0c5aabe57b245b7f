"""Clustering of strong pixels into spots (`xpg/spotcluster.py`), on the host: `cluster_spots` against XPG's own
accumulator's spots (tests/golden/spotcluster.npz, made by tests/golden/make_spotcluster_golden.py) on the strong
pixels of seeded runs: isolated spots, touching pairs (split at their separated peaks), and a ring of signal over every
frame (one cluster with hundreds of peaks: the huge-cluster rules), for two pixel-count ranges. Also `find_spots`'
glue for a frame stack (classifier, strong pixels read back, clustering) with the oracle's classifier on CPU tensors."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from xpg_b200 import spotcluster as SC

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
import make_spotcluster_golden as M  # noqa: E402

KEYS = ("x", "y", "z", "intensity", "npix", "zmin", "zmax")


@pytest.fixture(scope="module")
def gold():
    z = np.load(HERE / "golden" / "spotcluster.npz")
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("case", M.CASES, ids=lambda c: f"case{c[0]}")
def test_cluster_spots_matches_reference(case, gold):
    k, y, x, v, b, ny, nx = M.strong_pixels(*case)
    for ri, (mn, mx) in enumerate(M.RANGES):
        got = SC.cluster_spots(k, y, x, v, b, nx, ny, mn, mx, 3.0, 2)
        for key in KEYS:
            assert np.array_equal(got[key], gold[f"c{case[0]}_r{ri}_{key}"]), (case[0], ri, key)


def test_cluster_spots_empty_and_single():
    e = np.zeros(0, np.int32)
    got = SC.cluster_spots(e, e, e, e.astype(np.float32), e.astype(np.float32), 10, 10, 1, 100)
    assert all(got[k].size == 0 for k in KEYS)
    got = SC.cluster_spots([3], [4], [5], [10.0], [1.0], 10, 10, 1, 100)
    assert got["npix"].tolist() == [1] and got["x"].tolist() == [6.0] and got["z"].tolist() == [3.5]


def test_stack_glue_with_the_oracle_classifier():
    import torch
    from oracle import spotfind as OS
    from xpg_b200.spotfind import spots_of_stack
    rng = np.random.default_rng(2)
    img = rng.poisson(0.5, (6, 80, 90)).astype(np.float32)
    img[2:4, 30:34, 40:44] += 60.0
    img[1:3, 60:63, 10:13] += 40.0

    def finder(t, gain):
        s, m = OS.find(t.numpy(), gain)
        return torch.from_numpy(s), torch.from_numpy(m)
    got = spots_of_stack(torch.from_numpy(img), 1.0, first_frame=10, finder=finder, min_pix=4)
    s, m = OS.find(img, 1.0)
    k, y, x = np.nonzero(s)
    want = SC.cluster_spots(k + 10, y, x, img[k, y, x], m[k, y, x], 90, 80, 4, 1000000)
    assert len(got["x"]) >= 2
    for key in KEYS:
        assert np.array_equal(got[key], want[key]), key


def test_find_spots_matches_reference():
    """The drop-in `find_spots` (XPG's signature) against XPG's own run on the same image set: batches of 4 frames, a
    gap in the frame numbers, a static mask; the classifier here is the oracle's (on CPU tensors, bit-identical to
    XPG's classifier and to the device's), so what is compared is the batching, masking, read-back, clustering and
    the spot order (XPG's streaming clustering emits spots flush by flush)."""
    import torch
    import make_findspots_golden as F
    from oracle import spotfind as OS
    from oracle.gather import prepare_frame
    from xpg_b200.spotfind import find_spots
    raw = F.raw_frames()

    class Images:
        nx, ny, first, last = F.NX, F.NY, 1, F.NF

        def get(self, f):
            return prepare_frame(raw[f - 1], F.OVERLOAD)

    def finder(t, gain):
        s, m = OS.find(t.numpy(), gain)
        return torch.from_numpy(s), torch.from_numpy(m)
    got = find_spots(Images(), F.FRAMES, mask=F.static_mask(), verbose=False, finder=finder, device="cpu", **F.KW)
    want = np.load(HERE / "golden" / "findspots.npz")
    assert len(got) == want["x"].size > 100
    for key in KEYS:
        assert np.array_equal(getattr(got, key), want[key]), key


@pytest.mark.gpu
def test_find_spots_on_device_matches_reference():
    """The same run with the device classifier (`find_spots`' default): XPG's spots, in XPG's order."""
    import make_findspots_golden as F
    from oracle.gather import prepare_frame
    from xpg_b200.spotfind import find_spots
    raw = F.raw_frames()

    class Images:
        nx, ny, first, last = F.NX, F.NY, 1, F.NF

        def get(self, f):
            return prepare_frame(raw[f - 1], F.OVERLOAD)
    got = find_spots(Images(), F.FRAMES, mask=F.static_mask(), verbose=False, **F.KW)
    want = np.load(HERE / "golden" / "findspots.npz")
    for key in KEYS:
        assert np.array_equal(getattr(got, key), want[key]), key


@pytest.mark.parametrize("frames", [[3, 5, 4], [1, 2, 2, 3]])
def test_find_spots_refuses_frame_lists_that_are_not_increasing(frames):
    """Clustering all strong pixels at once links frames by number, which equals XPG's streaming clustering (closed at
    every break in the frame list) only when the frames increase: other lists are refused before any work."""
    from xpg_b200.spotfind import find_spots

    class Images:
        nx, ny, first, last = 8, 8, 1, 5

        def get(self, f):
            raise AssertionError("no frame is read")
    with pytest.raises(ValueError, match="strictly increasing"):
        find_spots(Images(), frames, verbose=False, finder=lambda t, g: None, device="cpu")
