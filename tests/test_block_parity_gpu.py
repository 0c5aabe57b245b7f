"""Parity on the benchmarked workload: one 360-frame phi block of the 16M-pixel sweep (430k reflections, boxes of
17-53 px and 17-65 frame bins, 5 x 5 profile regions), integrated by the drop-in `integrate()` from frames rendered on
the device, then at least 500 of its rows (every shoebox shape group, partners included) integrated again by the
restatement from the same raw frames, with the block's learnt profiles and adapted widths. Integers exact, floats
within tests/tolerance.py."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_config2_block_sample_matches_oracle():
    import torch
    import bench
    from oracle.blockcheck import check_rows, stratified_rows
    wl = bench.Workload("config2-block")
    res = wl.integrate(wl.source())
    p = wl.plan
    assert res.memory["parts"] == 1
    np.testing.assert_array_equal(res.refl["iz0"], p.iz0)
    assert np.isfinite(res.refl["iprf"]).all()
    rows = stratified_rows(p, np.arange(p.n), n_min=500)
    assert rows.size >= 500
    assert p.has_partner[rows].any() and (p.fb[rows] > 1).any()
    s = wl.spec
    worst, bad, info = check_rows(wl.crop, p, rows, res, 0, wl.exp.geom, wl.n_frames, s.ny, s.nx, s.overload,
                                  wl.model.gain)
    del wl, res
    torch.cuda.empty_cache()
    assert info["rows_fitted"] > 400
    assert all(v == 0 for v in bad.values()), (bad, worst)
