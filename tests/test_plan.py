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
                         spec.n_regions_xy, True, True, foreign_spots=G.foreign_of(case))
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


def test_foreign_spot_columns_match_reference():
    """Neighbour columns of a run given foreign spots (`xpg/integrate.py:304-327`): the reference's kernel inputs of
    every stored chunk row (8 neighbour columns, then 4 foreign-spot columns) equal the oracle planner's, float32 for
    float32; rows are matched by their predicted S."""
    case = "foreign"
    z = G.load(case)
    spec = G.case_inputs(case)[0]
    edges = z["edges"]
    model = IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m)
    p = plan_integration([spec.experiment()] * (len(edges) - 1), edges, model, float(z["dmin"]), 1e9,
                         (1, spec.nframes), 0.05, spec.n_regions_xy, True, True, foreign_spots=G.foreign_of(case))
    S32 = p.refl["S"].astype(np.float32)
    key = {tuple(s): j for j, s in enumerate(map(tuple, S32))}
    n_foreign_rows = 0
    for i in G.chunks(case):
        d, rc, nb, o1, o2 = G.chunk(case, i)
        assert nb["x"].shape[1] == 12
        for r in range(rc["S"].shape[0]):
            j = key[tuple(np.asarray(rc["S"][r], np.float32))]
            for k in ("x", "y", "z", "sx", "sz"):
                np.testing.assert_array_equal(p.nb[k][j], nb[k][r], err_msg=f"chunk {i} row {r} nb{k}")
            n_foreign_rows += int((nb["x"][r, 8:] > -1e5).any())
    assert n_foreign_rows > 10
