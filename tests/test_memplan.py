"""Device-memory planning (xpg_b200.memplan, the device counterpart of XPG's `_plan_passes` / `_split_blocks`,
xpg/shoebox.py:134-196 and xpg/integrate.py:592-626): CPU checks on a golden sweep's plan."""
from __future__ import annotations

import numpy as np

import golden_io as G
from oracle.plan import plan_integration
from xpg_b200 import memplan as M
from xpg_b200.plan import IntegrationModel


def _plan(case):
    z = G.load(case)
    spec = G.case_inputs(case)[0]
    edges = z["edges"]
    exps = [spec.experiment()] * (len(edges) - 1)
    model = IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m)
    return plan_integration(exps, edges, model, float(z["dmin"]), 1e9, (1, spec.nframes), 0.05, spec.n_regions_xy,
                            True, True), exps, spec.nframes


def test_fit_keeps_a_plan_that_fits():
    p, exps, nf = _plan("adaptive")
    q, e, info = M.fit(p, exps, nf, 0, 1e15)
    assert q is p and e is exps and info["parts"] == 1


def test_fit_splits_blocks_into_parts_of_consecutive_phi():
    p, exps, nf = _plan("adaptive")
    w = M.row_bytes(p)
    one, big = M.peak_bytes(p.blocks_refl, p.need_lo, p.need_hi, w, nf)
    q, e, info = M.fit(p, exps, nf, 0, 0.6 * one)
    assert info["parts"] >= 2 and info["peak"] < one
    assert len(e) == len(q.blocks_refl) == len(info["parent"])
    rows = np.concatenate(q.blocks_refl)
    assert np.array_equal(np.sort(rows), np.arange(p.n))               # every row in exactly one part
    z = p.refl["z"]
    for b in range(len(p.blocks_refl)):
        mine = [q.blocks_refl[k] for k, par in enumerate(info["parent"]) if par == b]
        for a, c in zip(mine, mine[1:]):                               # parts follow each other in phi
            assert z[a].max() <= z[c].min()
        sizes = [w[r].sum() for r in mine]
        assert max(sizes) <= 1.6 * min(sizes)                          # about equal bytes
        for k, r in ((k, q.blocks_refl[k]) for k, par in enumerate(info["parent"]) if par == b):
            assert q.need_lo[k] == int(p.zstart[r].min()) and q.need_hi[k] == int(p.zend[r].max())


def test_split_blocks_matches_the_reference_rule():
    """The parts follow XPG's rule: rows ordered by z, cut where the cumulative bytes pass k equal shares."""
    p, exps, nf = _plan("config1")
    w = M.row_bytes(p)
    parts, parent = M.split_blocks(p.blocks_refl, p.refl["z"], w, 3)
    rows = p.blocks_refl[0]
    o = rows[np.argsort(p.refl["z"][rows], kind="stable")]
    c = np.cumsum(w[o])
    cuts = [0] + [int(np.searchsorted(c, c[-1] * f, side="right")) for f in (1 / 3, 2 / 3)] + [o.size]
    for k in range(3):
        np.testing.assert_array_equal(parts[k], np.sort(o[cuts[k]:cuts[k + 1]]))


def test_passes_group_blocks_m_apart_when_parts_do_not_fit():
    """Blocks whose boxes are deeper than the blocks themselves stay open together even in parts: then the blocks
    go in passes over the frames, m apart in phi (XPG's `_plan_passes` grouping), the fewest that fit."""
    p, exps, nf = _plan("adaptive")
    w = M.row_bytes(p)
    one, big = M.peak_bytes(p.blocks_refl, p.need_lo, p.need_hi, w, nf)
    passes, pk = M.split_passes(p, w, nf, big)
    assert len(passes) == 2 and sorted(sum(passes, [])) == [0, 1] and pk <= big
    q, e, info = M.fit(p, exps, nf, 0, 0.55 * one)
    assert "passes" in info and info["peak"] < one
    assert sorted(sum(info["passes"], [])) == list(range(len(q.blocks_refl)))
    q2, e2, info2 = M.fit(p, exps, nf, 0, 0.55 * one, allow_passes=False)
    assert "passes" not in info2
