"""Oracle of the integration plan: TEST INFRASTRUCTURE (see oracle/__init__.py).

The reference's host planning restated in float64 numpy (`xpg/integrate.py:101-122` predictions per phi block,
`:164-172` neighbour lists, `:222-370` boxes, partners and regions; `xpg/geometry.py:468-545` predictions), operation
for operation, so that every integer it produces equals XPG's. Pinned against the reference's plans of the golden
sweeps (tests/test_plan.py); the device planner (xpg_b200.plan) is checked against it.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree
from scipy.special import erf

from xpg_b200.geometry import PIX0, centring_allowed, generate_hkl, predict_reflections
from xpg_b200.plan import (BIN_MAX, BIN_SLOTS, DZ_BUCKETS, K_NEIGHBOURS, N_BOX, N_BOX_Z, N_FG, SUPERPIXEL,
                           SUPERPIXEL_MAX, XY_BUCKETS, IntegrationModel, Plan, depth_bucket)


def predict_blocks(exps_by_block, block_edges, dmin, dmax, z_lo, z_hi, minimum_zeta=0.05, lattice_of=None,
                   allowed=centring_allowed):
    """Predictions of every phi block with its own experiment (`xpg/integrate.py:101-122`). Block b of the flat
    list covers block_edges[b % n], block_edges[b % n + 1]; lattice_of[b] is its lattice id."""
    parts = []
    n_edges = len(block_edges) - 1
    for b, exp in enumerate(exps_by_block):
        za, zb = block_edges[b % n_edges], block_edges[b % n_edges + 1]
        hkl = generate_hkl(exp.crystal.Astar, dmin, dmax)
        hkl = hkl[allowed(hkl, exp.crystal.space_group)]
        pr = predict_reflections(exp.geom, exp.crystal.Astar, dmin, dmax, z_range=(za, zb), hkl=hkl)
        pr["block"] = np.full(pr["x"].size, b, np.int32)
        pr["lattice"] = np.full(pr["x"].size, 0 if lattice_of is None else lattice_of[b], np.int32)
        parts.append(pr)
    res = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    g = exps_by_block[0].geom
    e1 = np.cross(res["S"], g.s0)
    e1 /= np.maximum(np.linalg.norm(e1, axis=1, keepdims=True), 1e-12)
    res["zeta_k"] = e1 @ g.axis
    ok = (np.abs(res["zeta_k"]) >= minimum_zeta) & (res["x"] >= 0.5) & (res["x"] < g.nx + 0.5) & \
         (res["y"] >= 0.5) & (res["y"] < g.ny + 0.5) & (res["z"] >= z_lo) & (res["z"] < z_hi)
    return {k: v[ok] for k, v in res.items()}


def neighbour_lists(x, y, z, sx, sz, k=K_NEIGHBOURS):
    """k nearest reflections within 4 N_FG in (x / sx, y / sx, z / sz) (`xpg/integrate.py:164-172`)."""
    pts = np.c_[x / sx, y / sx, z / sz]
    d, j = cKDTree(pts).query(pts, k=k + 1, distance_upper_bound=4.0 * N_FG, workers=-1)
    j, d = j[:, 1:], d[:, 1:]
    has = np.isfinite(d)
    return np.where(has, j, 0), has, np.where(has, d, np.inf)


def plan_integration(exp_blocks, block_edges, model, dmin, dmax=1e9, frames=(1, 1), minimum_zeta=0.05,
                     n_regions_xy=3, adaptive=True, deconvolve_overlaps=True, lattice_of=None, foreign_spots=None,
                     n_foreign=4, allowed=centring_allowed):
    """Predictions and shoebox plan of a sweep (`xpg/integrate.py:222-370`)."""
    g0 = exp_blocks[0].geom
    f_first, f_last = frames
    z_lo, z_hi = f_first - 1.0, float(f_last)
    refl = predict_blocks(exp_blocks, block_edges, dmin, dmax, z_lo, z_hi, minimum_zeta, lattice_of, allowed)
    widen = 1.3 if adaptive else 1.0
    box = (IntegrationModel(model.sigma_d * widen, model.sigma_m).box(g0) if not model.box_xy else model.box_xy)
    half = box // 2
    sd = np.radians(model.sigma_d)
    # depth: N_BOX_Z sigma of the rocking curve each side; very wide reflections binned by fb frames
    sz_frames = model.sigma_m / np.abs(refl["zeta_k"]) / abs(g0.osc)
    hz = np.ceil(N_BOX_Z * sz_frames + 0.5).astype(int)
    hmax = (max(DZ_BUCKETS) - 1) // 2
    wide = hz > hmax
    fb = np.where(wide, np.clip(np.ceil((2 * hz + 1) / BIN_SLOTS), 2, BIN_MAX), 1).astype(int)
    hz = np.where(wide, np.minimum(np.ceil(N_BOX_Z * sz_frames / fb + 0.5).astype(int), (BIN_SLOTS - 1) // 2),
                  hz).astype(int)
    trunc = wide & (np.ceil(N_BOX_Z * sz_frames / fb + 0.5) > (BIN_SLOTS - 1) // 2)
    iz_c = np.floor(refl["z"] - (fb - 1) / 2.0).astype(int)
    iz0 = iz_c - hz * fb
    dz = 2 * hz + 1
    Dz = depth_bucket(dz)
    zc = refl["z"]
    cov = 0.5 * (erf((iz0 + dz * fb - zc) / (np.sqrt(2) * sz_frames)) - erf((iz0 - zc) / (np.sqrt(2) * sz_frames)))
    refl["coverage"] = np.where(trunc, np.clip(cov, 0, 1), 1.0).astype(np.float32)
    keep = Dz > 0
    info = dict(n_predicted=int(refl["x"].size), n_wide=int(wide.sum()), n_trunc=int(trunc.sum()), box=box)
    refl = {k: v[keep] for k, v in refl.items()}
    iz0, dz, Dz, fb = iz0[keep], dz[keep], Dz[keep], fb[keep]
    n = refl["x"].size
    # box side from the local footprint of sigma_D (distance, obliquity), bucketed
    if model.box_xy:
        bxs = np.full(n, box, int)
        spx = None
    else:
        Xv = g0.pixel_to_lab(refl["x"], refl["y"])
        Lr = np.linalg.norm(Xv, axis=1)
        cosr = np.abs(Xv @ g0.ed3) / Lr
        spx = Lr * np.radians(model.sigma_d * widen) / min(g0.qx, g0.qy) / np.maximum(cosr, 0.4)
        spx = np.sqrt(spx ** 2 + 1.0 / 12.0)
        need = 2 * np.maximum(np.ceil(N_BOX * spx).astype(int) + 1, 2) + 1
        xyb = np.array([b_ for b_ in XY_BUCKETS if b_ < box] + [box])
        bxs = xyb[np.minimum(np.searchsorted(xyb, need), len(xyb) - 1)]
    pxs = np.ones(n, int)
    if SUPERPIXEL > 0 and not model.box_xy and n:
        pxs = np.clip(np.floor(spx / SUPERPIXEL), 1, SUPERPIXEL_MAX).astype(int)
        need_s = 2 * np.maximum(np.ceil(N_BOX * spx / pxs).astype(int) + 1, 2) + 1
        bxs = np.where(pxs > 1, xyb[np.minimum(np.searchsorted(xyb, need_s), len(xyb) - 1)], bxs)
    halfs = bxs // 2
    ix0 = np.floor(refl["x"] - PIX0 + 0.5).astype(int) // pxs - halfs
    iy0 = np.floor(refl["y"] - PIX0 + 0.5).astype(int) // pxs - halfs
    # neighbour ellipsoids (N_FG sigma) and overlap partners
    Xlen = np.linalg.norm(g0.pixel_to_lab(refl["x"], refl["y"]), axis=1)
    sx_px = np.maximum(Xlen * sd / g0.qx, 0.5) * N_FG
    sz_f = np.sqrt((model.sigma_m / np.abs(refl["zeta_k"])) ** 2 + (g0.osc ** 2) / 12.0) / abs(g0.osc) * N_FG
    if n:
        nbj, nbh, nbd = neighbour_lists(refl["x"], refl["y"], refl["z"], sx_px.mean(), sz_f.mean())
    else:
        nbj = np.zeros((0, K_NEIGHBOURS), int)
        nbh = np.zeros((0, K_NEIGHBOURS), bool)
        nbd = np.zeros((0, K_NEIGHBOURS))
    has_partner = (nbh[:, 0] & (nbd[:, 0] < 2.0)) if deconvolve_overlaps else np.zeros(len(nbd), bool)
    nb = dict(x=np.where(nbh, refl["x"][nbj], -1e6).astype(np.float32),
              y=np.where(nbh, refl["y"][nbj], -1e6).astype(np.float32),
              z=np.where(nbh, refl["z"][nbj], -1e6).astype(np.float32),
              sx=np.where(nbh, sx_px[nbj], 1.0).astype(np.float32),
              sz=np.where(nbh, sz_f[nbj], 1.0).astype(np.float32))
    if foreign_spots is not None and len(foreign_spots[0]) and n:
        fx, fy, fz = (np.asarray(a, float) for a in foreign_spots)
        sxm, szm = float(sx_px.mean()), float(sz_f.mean())
        ft = cKDTree(np.c_[fx / sxm, fy / sxm, fz / szm])
        d_f, j_f = ft.query(np.c_[refl["x"] / sxm, refl["y"] / sxm, refl["z"] / szm], k=n_foreign + 2,
                            distance_upper_bound=4.0 * N_FG)
        d_f, j_f = np.atleast_2d(d_f), np.atleast_2d(j_f)
        hf = np.isfinite(d_f) & (d_f > 2.5 / N_FG)
        order_f = np.argsort(np.where(hf, d_f, np.inf), axis=1)[:, :n_foreign]
        rows_f = np.arange(d_f.shape[0])[:, None]
        hf, j_f = hf[rows_f, order_f], np.where(np.isfinite(d_f), j_f, 0)[rows_f, order_f]
        rad = 2.0 / N_FG
        nb["x"] = np.concatenate([nb["x"], np.where(hf, fx[j_f], -1e6).astype(np.float32)], 1)
        nb["y"] = np.concatenate([nb["y"], np.where(hf, fy[j_f], -1e6).astype(np.float32)], 1)
        nb["z"] = np.concatenate([nb["z"], np.where(hf, fz[j_f], -1e6).astype(np.float32)], 1)
        nb["sx"] = np.concatenate([nb["sx"], np.full(hf.shape, sxm * rad, np.float32)], 1)
        nb["sz"] = np.concatenate([nb["sz"], np.full(hf.shape, szm * rad, np.float32)], 1)
    rx = np.clip((refl["x"] / g0.nx * n_regions_xy).astype(int), 0, n_regions_xy - 1)
    ry = np.clip((refl["y"] / g0.ny * n_regions_xy).astype(int), 0, n_regions_xy - 1)
    region = (ry * n_regions_xy + rx).astype(np.int32)
    nblocks = len(exp_blocks)
    blk = refl["block"]
    zstart = np.maximum(iz0, f_first - 1)
    zend = np.minimum(iz0 + dz * fb - 1, f_last - 1)
    order = np.argsort(blk, kind="stable")
    blocks_refl = [order[blk[order] == b] for b in range(nblocks)]
    need_lo = [int(zstart[r].min()) if r.size else 10 ** 9 for r in blocks_refl]
    need_hi = [int(zend[r].max()) if r.size else -1 for r in blocks_refl]
    return Plan(refl=refl, iz0=iz0, dz=dz, fb=fb, Dz=Dz, bx=bxs.astype(int), pxs=pxs, ix0=ix0, iy0=iy0,
                region=region, has_partner=has_partner, partner=nbj[:, 0] if n else np.zeros(0, int), nb=nb,
                overlap=has_partner.copy(), nreg=n_regions_xy * n_regions_xy, box=box, blocks_refl=blocks_refl,
                need_lo=need_lo, need_hi=need_hi, zstart=zstart, zend=zend, info=info)
