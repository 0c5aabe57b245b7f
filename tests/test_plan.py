"""Oracle planner pinned (CPU): its predictions and every integer of its shoebox plan equal the reference's."""
from __future__ import annotations

import numpy as np
import pytest

import golden_io as G
from oracle.plan import plan_integration
from xpg_b200.plan import IntegrationModel


@pytest.mark.parametrize("case", G.CASES)
def test_plan_matches_reference(case):
    z = G.load(case)
    spec, tmpl, mask, excl = G.case_inputs(case)
    exp = spec.experiment()
    edges = z["edges"]
    model = IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m)
    p = plan_integration([exp] * (len(edges) - 1), edges, model, float(z["dmin"]), 1e9, (1, spec.nframes), 0.05,
                         spec.n_regions_xy, True, True)
    out = {k[4:]: v for k, v in z.items() if k.startswith("out_")}
    assert p.n == len(out["x"])
    assert np.array_equal(p.refl["hkl"], out["hkl"])
    for k in ("x", "y", "z", "phi"):
        np.testing.assert_allclose(p.refl[k], out[k], rtol=0, atol=1e-9)
    np.testing.assert_allclose(p.refl["S"], out["S"], rtol=0, atol=1e-12)
    assert np.array_equal(p.iz0, out["iz0"])
    assert np.array_equal(p.dz, out["dz"])
    assert np.array_equal(p.fb, out["fb"])
    assert np.array_equal(p.region, out["region"])
    assert np.array_equal(p.ix0 * p.pxs, out["ix0"])
    assert np.array_equal(p.iy0 * p.pxs, out["iy0"])
    assert np.array_equal(p.overlap, out["overlap"])
    if "pxs" in out:
        assert np.array_equal(p.pxs, out["pxs"])
    else:
        assert (p.pxs == 1).all()
    np.testing.assert_array_equal(p.refl["coverage"], out["coverage"])
