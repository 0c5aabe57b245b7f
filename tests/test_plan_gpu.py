"""Device planner parity (GPU): the plan from libxpgi.so's planning entry points (predictions, shoebox rules,
neighbour search) equals the reference's on the golden sweeps, and the oracle planner's on the config-2 block
(430k reflections), on segmented / parallax / distortion-table detectors, with several blocks and lattices, and with
a caller's own absence rule. Integers are compared exactly; float64 predictions to 1e-12 relative (CUDA's and the
host's transcendental functions may differ in the last bit; detector positions to 1e-9 pixels, as the reference's
own planner is pinned)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

import golden_io as G
from oracle import plan as OPL
from xpg_b200 import native as N
from xpg_b200 import synth
from xpg_b200.geometry import Experiment, Panel, random_orientation
from xpg_b200.plan import IntegrationModel, plan_integration

pytestmark = pytest.mark.gpu

INTS = ("iz0", "dz", "fb", "Dz", "bx", "pxs", "ix0", "iy0", "region", "zstart", "zend", "has_partner", "overlap",
        "partner")
F64 = ("x", "y", "z", "phi", "zeta", "polarization", "zeta_k")


def assert_same_plan(p, q):
    """p: device plan, q: oracle plan."""
    assert p.n == q.n
    assert p.info == q.info
    for k in ("hkl", "block", "lattice"):
        np.testing.assert_array_equal(p.refl[k], q.refl[k], err_msg=k)
    for k in F64:                           # positions carry the rounding of their (thousand-pixel) offsets
        np.testing.assert_allclose(p.refl[k], q.refl[k], rtol=1e-12, atol=1e-9 if k in ("x", "y", "z", "phi") else
                                   1e-12, err_msg=k)
    np.testing.assert_allclose(p.refl["S"], q.refl["S"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(p.refl["coverage"], q.refl["coverage"], rtol=1e-6, atol=0)
    for k in INTS:
        np.testing.assert_array_equal(getattr(p, k), getattr(q, k), err_msg=k)
    for k in ("x", "y", "z", "sx", "sz"):
        np.testing.assert_allclose(p.nb[k], q.nb[k], rtol=1e-6, atol=0, err_msg="nb" + k)
    assert p.need_lo == q.need_lo and p.need_hi == q.need_hi
    for a, b in zip(p.blocks_refl, q.blocks_refl):
        np.testing.assert_array_equal(a, b)


def both(exps, edges, model, dmin, frames, n_regions_xy=3, **kw):
    args = (exps, edges, model, dmin, 1e9, frames, 0.05, n_regions_xy, True, True)
    return plan_integration(*args, **kw), OPL.plan_integration(*args, **kw)


@pytest.mark.parametrize("case", G.CASES)
def test_device_plan_matches_reference(case):
    z = G.load(case)
    spec, tmpl, mask, excl = G.case_inputs(case)
    edges = z["edges"]
    model = IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m)
    p = plan_integration([spec.experiment()] * (len(edges) - 1), edges, model, float(z["dmin"]), 1e9,
                         (1, spec.nframes), 0.05, spec.n_regions_xy, True, True, foreign_spots=G.foreign_of(case))
    out = {k[4:]: v for k, v in z.items() if k.startswith("out_")}
    assert p.n == len(out["x"])
    np.testing.assert_array_equal(p.refl["hkl"], out["hkl"])
    for k in ("x", "y", "z", "phi"):
        np.testing.assert_allclose(p.refl[k], out[k], rtol=0, atol=1e-9)
    np.testing.assert_allclose(p.refl["S"], out["S"], rtol=0, atol=1e-12)
    for k in ("iz0", "dz", "fb", "region", "overlap"):
        np.testing.assert_array_equal(getattr(p, k), out[k], err_msg=k)
    np.testing.assert_array_equal(p.ix0 * p.pxs, out["ix0"])
    np.testing.assert_array_equal(p.iy0 * p.pxs, out["iy0"])
    np.testing.assert_array_equal(p.pxs, out["pxs"] if "pxs" in out else np.ones(p.n, np.int64))
    np.testing.assert_allclose(p.refl["coverage"], out["coverage"], rtol=1e-6, atol=0)


def test_device_plan_matches_oracle_config2_block():
    s = synth.config2()
    model = IntegrationModel(sigma_d=s.sigma_d, sigma_m=s.sigma_m)
    p, q = both([s.experiment()], np.array([0.0, 360.0]), model, s.resolution_limit(), (1, 372), s.n_regions_xy)
    assert p.n > 400_000
    assert_same_plan(p, q)


def _small(**kw):
    s = synth.config1(**kw)
    return s, IntegrationModel(sigma_d=s.sigma_d, sigma_m=s.sigma_m)


def test_device_plan_segmented_parallax_distortion():
    s, model = _small(sensor_thickness=0.45, mu=3.0)
    exp = s.experiment()
    g = exp.geom
    tilt = np.array([0.0, np.cos(0.01), np.sin(0.01)])
    segs = [Panel(1, s.nx, 1, 500), Panel(1, s.nx, 511, s.ny, orgy=0.3, distance=0.2, ey=tilt)]
    yy, xx = np.mgrid[0:s.ny, 0:s.nx]
    geo = (0.4 * np.sin(xx / 97.0) * np.cos(yy / 61.0), -0.3 * np.cos(xx / 53.0 + yy / 89.0))
    for kw in (dict(segments=segs), dict(geo_corr=geo), dict(segments=segs, geo_corr=geo)):
        e = Experiment(g.copy(**kw), exp.crystal)
        p, q = both([e], np.array([0.0, 100.0]), model, s.resolution_limit(), (1, s.nframes))
        assert p.n > 1000
        assert_same_plan(p, q)


def test_device_plan_blocks_lattices_and_own_absences():
    s, model = _small()
    exp = s.experiment()
    other = Experiment(exp.geom, type(exp.crystal)(U=random_orientation(np.random.default_rng(7)),
                                                   cell=np.array(s.cell, float), space_group="C 2 2 21"))
    edges = np.array([0.0, 30.0, 65.0, 100.0])
    p, q = both([exp] * 3 + [other] * 3, edges, model, s.resolution_limit(), (1, s.nframes),
                lattice_of=[0, 0, 0, 1, 1, 1])
    assert set(np.unique(p.refl["lattice"])) == {0, 1}
    assert_same_plan(p, q)
    odd_l = lambda hkl, sg: hkl[:, 2] % 2 == 1
    p, q = both([exp], np.array([0.0, 100.0]), model, s.resolution_limit(), (1, s.nframes), allowed=odd_l)
    assert (p.refl["hkl"][:, 2] % 2 == 1).all()
    assert_same_plan(p, q)


def test_knn_matches_kdtree():
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(5)
    n, k = 60_000, 8
    x, y, z = rng.uniform(0, 9000, n), rng.uniform(0, 7000, n), rng.uniform(0, 100, n)   # ~5 within reach
    sx, sz = 7.5, 1.25
    pts = np.c_[x / sx, y / sx, z / sz]
    d_ref, j_ref = cKDTree(pts).query(pts, k=k + 1, distance_upper_bound=12.0)
    d_ref, j_ref = d_ref[:, 1:], j_ref[:, 1:]
    has = np.isfinite(d_ref)
    lib = N.load()
    t = {a: torch.as_tensor(v).cuda() for a, v in (("x", x), ("y", y), ("z", z))}
    q = N.XiKnn()
    q.n, q.x, q.y, q.z, q.sx, q.sz, q.radius, q.k = n, N.ptr(t["x"]), N.ptr(t["y"]), N.ptr(t["z"]), sx, sz, 12.0, k
    q.lo[:] = [0.0, 0.0, 0.0]
    q.hi[:] = [9000 / sx, 7000 / sx, 100 / sz]
    ws = torch.empty(int(lib.xi_knn_workspace(C.byref(q))), dtype=torch.uint8, device="cuda")
    nbj = torch.empty((n, k), dtype=torch.int32, device="cuda")
    nbd = torch.empty((n, k), dtype=torch.float64, device="cuda")
    N.check(lib.xi_knn(C.byref(q), N.ptr(ws), ws.numel(), N.ptr(nbj), N.ptr(nbd), N.stream_handle()), "xi_knn")
    j, d = nbj.cpu().numpy(), nbd.cpu().numpy()
    assert has.sum() > n                         # some points have neighbours, some have fewer than k
    assert (~has).sum() > 0
    np.testing.assert_array_equal(np.isfinite(d), has)
    np.testing.assert_array_equal(np.where(has, j, 0), np.where(has, j_ref, 0))
    np.testing.assert_array_equal(d[has], d_ref[has])
