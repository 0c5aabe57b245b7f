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
    q, e, info = M.fit(p, exps, nf, 0, 0.6 * one, allow_passes=False)     # frames read once: parts only
    assert info["parts"] >= 2 and info["peak"] < one and "passes" not in info
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


def test_passes_group_blocks_m_apart():
    """Blocks open together that do not fit go in passes over the frames, m apart in phi (XPG's `_plan_passes`
    grouping), the fewest that fit, before any block is split (xpg/integrate.py:598-622)."""
    p, exps, nf = _plan("adaptive")
    w = M.row_bytes(p)
    one, big = M.peak_bytes(p.blocks_refl, p.need_lo, p.need_hi, w, nf)
    passes, pk = M.split_passes([w[r].sum() for r in p.blocks_refl], p.need_lo, p.need_hi, [0, 0], nf, big)
    assert len(passes) == 2 and sorted(sum(passes, [])) == [0, 1] and pk <= big
    q, e, info = M.fit(p, exps, nf, 0, 0.55 * one)
    assert "passes" in info and info["peak"] < one
    assert info["parts"] == 1 and q is p          # XPG's order: whole blocks in passes before any split
    assert sorted(sum(info["passes"], [])) == list(range(len(q.blocks_refl)))
    q2, e2, info2 = M.fit(p, exps, nf, 0, 0.55 * one, allow_passes=False)
    assert "passes" not in info2


def test_passes_over_parts_when_rows_wide_in_phi_keep_every_part_open():
    """One phi block whose rows include some wide in phi (binned boxes spanning the whole sweep): every part of the
    block then reaches from the first frame to the last, so no split lowers the peak; the parts go in passes over
    the frames instead, the fewest parts whose passes fit, every row in exactly one part of one pass."""
    from dataclasses import replace
    p, exps, nf = _plan("config1")
    assert len(p.blocks_refl) == 1
    zs, ze = p.zstart.copy(), p.zend.copy()
    z = p.refl["z"]
    o = np.argsort(z, kind="stable")
    wide = o[::50]                                              # a few rows in every part span the sweep
    zs[wide], ze[wide] = 0, nf - 1
    p = replace(p, zstart=zs, zend=ze, need_lo=[0], need_hi=[nf - 1])
    w = M.row_bytes(p)
    one, _ = M.peak_bytes(p.blocks_refl, p.need_lo, p.need_hi, w, nf)
    parts, parent = M.split_blocks(p.blocks_refl, z, w, 8)
    lo = [int(zs[r].min()) for r in parts]
    hi = [int(ze[r].max()) for r in parts]
    assert M.peak_bytes(parts, lo, hi, w, nf)[0] == one                # parts alone do not help
    q, e, info = M.fit(p, exps, nf, 0, 0.6 * one)
    assert info["parts"] >= 2 and len(info["passes"]) >= 2 and info["peak"] <= 0.6 * one
    assert sorted(sum(info["passes"], [])) == list(range(len(q.blocks_refl)))
    rows = np.concatenate(q.blocks_refl)
    assert np.array_equal(np.sort(rows), np.arange(p.n))
    q2, e2, info2 = M.fit(p, exps, nf, 0, 0.6 * one, allow_passes=False)
    # frames read once: the wide rows go in a part of their own, the others in parts of consecutive phi
    assert "passes" not in info2 and info2.get("wide_apart") and info2["peak"] <= 0.6 * one
    assert np.array_equal(np.sort(np.concatenate(q2.blocks_refl)), np.arange(p.n))
    assert any(np.isin(wide, r).all() for r in q2.blocks_refl)     # every planted wide row in the wide part


def test_passes_by_lattice_first():
    """Blocks of two lattices over the same frames: the first pass grouping tried after one pass is by lattice
    (xpg/shoebox.py:163-170), then m apart in phi within each lattice."""
    rng = np.random.default_rng(3)
    blocks = [np.arange(10 * b, 10 * b + 10) for b in range(6)]          # lattice 0: blocks 0-2, lattice 1: 3-5
    lo = [0, 100, 200, 0, 100, 200]
    hi = [150, 250, 299, 150, 250, 299]
    w = rng.uniform(1, 2, 60)
    one = M.peak_bytes(blocks, lo, hi, w, 300)[0]
    nbytes = [w[r].sum() for r in blocks]
    passes, pk = M.split_passes(nbytes, lo, hi, [0, 0, 0, 1, 1, 1], 300, 0.6 * one)
    assert passes == [[0, 1, 2], [3, 4, 5]] and pk <= 0.6 * one
    passes, pk = M.split_passes(nbytes, lo, hi, [0, 0, 0, 1, 1, 1], 300, 0.3 * one)
    assert len(passes) == 4 and sorted(sum(passes, [])) == list(range(6))
    assert all(len({b // 3 for b in q}) == 1 for q in passes)           # each pass holds one lattice


def test_row_bytes_table_matches_the_formula():
    """The table lookup of row_bytes gives the formula's bytes for every bucket combination, and the formula itself
    answers values beyond the table."""
    from types import SimpleNamespace
    rng = np.random.default_rng(9)
    n = 20000
    Dz = rng.choice([3, 5, 9, 17, 33, 65], n).astype(np.int32)
    bx = rng.choice([9, 13, 17, 23, 31, 41, 55, 73, 97], n).astype(np.int32)
    fb = np.where(rng.random(n) < 0.1, rng.integers(2, 9, n), 1).astype(np.int32)
    p = SimpleNamespace(Dz=Dz, bx=bx, fb=fb)
    np.testing.assert_array_equal(M.row_bytes(p), M._bytes_of(Dz, bx, fb > 1))
    q = SimpleNamespace(Dz=np.array([130, 5]), bx=np.array([9, 200]), fb=np.array([1, 3]))
    np.testing.assert_array_equal(M.row_bytes(q), M._bytes_of(q.Dz, q.bx, q.fb > 1))
