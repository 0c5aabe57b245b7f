"""XPG's inner kernel surface (make_kernels) on the B200 kernels reproduces the reference's outputs on a golden
chunk, through the same dict interface."""
from __future__ import annotations

import numpy as np
import pytest

import golden_io as G
import tolerance as T

pytestmark = pytest.mark.gpu


def test_make_kernels_surface_matches_reference():
    from xpg_b200.kernels import detector_consts, make_kernels
    case = "crowded"
    spec, tmpl, mask, excl = G.case_inputs(case)
    d, rc, nb, o1, o2 = G.chunk(case, 0)
    Dz, Dy, Dx = (int(v) for v in d["shape"])
    p1, acc, p2 = make_kernels(Dz, Dy, Dx, spec.n_regions_xy ** 2)
    det = detector_consts(spec.geometry(), tmpl)
    r1 = p1(d["sb"], rc, det, d["axis"], d["s0"], d["frames_phi0"], d["osc"], d["sd"], d["sm"], d["gain"], None, nb,
            d["rcw"])
    h1 = {k: v.cpu().numpy() for k, v in r1.items() if not k.startswith("_")}
    for j in range(d["sb"].shape[0]):
        ctx = {k: o1[k][j] for k in o1}
        for k in ("n_over", "n_fg_masked", "n_fg_nb"):
            assert int(h1[k][j]) == int(o1[k][j]), (j, k)
        for k in ("bg", "isum", "vsum", "img2", "J", "u1", "u2"):
            ok, w = T.within(k, h1[k][j], o1[k][j], ctx)
            assert ok, (j, k, w)
    sel = np.ones(d["sb"].shape[0], bool)
    num, den = acc(r1["img2"], r1["all_valid2"], r1["J"], r1["u1"], r1["u2"], rc["region"], r1["isum"], sel,
                   r1["seff"])
    assert float(den.sum()) > 0
    pix = {k: r1[k] for k in ("zeta", "J", "u1", "u2", "seff")}
    r2 = p2(d["sb"], rc, det, d["axis"], d["s0"], d["frames_phi0"], d["osc"], d["p2_sd"], d["p2_sm"], d["p2_gain"],
            d["prof"], r1["bg"], r1["nbg"], nb, d["p2_rcw"], pix)
    h2 = {k: v.cpu().numpy() for k, v in r2.items()}
    for j in range(d["sb"].shape[0]):
        ctx = {k: o2[k][j] for k in o2}
        for k in ("iprf", "vprf", "p_total", "p_fg"):
            ok, w = T.within(k, h2[k][j], o2[k][j], ctx)
            assert ok, (j, k, w)
