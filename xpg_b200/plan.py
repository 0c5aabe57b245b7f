"""Planning of an integration run on the device: predictions per phi block, shoebox boxes (depth, phi binning,
side, super-pixels, origin), neighbour lists, overlap partners and detector regions (`xpg/integrate.py:222-370`).

XPG plans in numpy on the host. Here the per-reflection float64 arithmetic runs in libxpgi.so (`xi_predict_count` /
`xi_predict_write` over the Miller-index grid, `xi_plan_boxes`, `xi_knn`) in numpy's operation order, so that every
integer of the plan (boxes, buckets, frame ranges, neighbours) is XPG's; the host computes the per-geometry
constants with the same numpy expressions as the reference, the two means of the neighbour scales, and the block
bookkeeping. The result is a `Plan` of host arrays (the device columns stay available in `Plan.dev`).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import native as N
from .device import TIMER, d2h, h2d
from .geometry import centring_allowed, generate_hkl, unit

N_FG = 3.0
N_BOX = 5.0
N_BOX_Z = 4.0
DZ_BUCKETS = (3, 5, 9, 17, 33, 65)
BIN_SLOTS = 33
BIN_MAX = 8
XY_BUCKETS = (9, 13, 17, 23, 31, 41, 55, 73, 97)
SUPERPIXEL = 2.5
SUPERPIXEL_MAX = 4
K_NEIGHBOURS = 8


@dataclass
class IntegrationModel:
    """Spot widths of an integration run (`xpg/integrate.py:60-79`): e.s.d.s in degrees, detector gain and an
    optional fixed box side."""
    sigma_d: float
    sigma_m: float
    gain: float = 1.0
    box_xy: int = 0

    def box(self, geom, dmin=None):
        """Odd box side covering N_BOX sigma_D at the most oblique detector corner."""
        if self.box_xy:
            return self.box_xy
        corners = geom.pixel_to_lab(np.array([0.5, geom.nx + .5, 0.5, geom.nx + .5]),
                                    np.array([0.5, 0.5, geom.ny + .5, geom.ny + .5]))
        L = np.linalg.norm(corners, axis=1).max()
        cos2t = geom.distance / L
        spx = L * np.radians(self.sigma_d) / min(geom.qx, geom.qy) / max(cos2t, 0.4)
        spx = math.sqrt(spx ** 2 + 1.0 / 12.0)
        h = int(math.ceil(N_BOX * spx)) + 1
        return 2 * max(h, 2) + 1


def depth_bucket(dz):
    """Smallest DZ_BUCKETS entry >= dz, -1 beyond the deepest (`xpg/integrate.py:157-161`)."""
    b = np.asarray(DZ_BUCKETS)
    k = np.searchsorted(b, dz, side="left")
    return np.where(k < len(b), b[np.minimum(k, len(b) - 1)], -1).astype(int)


@dataclass
class Plan:
    """Everything the device needs to integrate a sweep, per reflection (after the depth-bucket cut)."""
    refl: dict                      # predictions (x, y, z, phi, S, zeta_k, block, lattice, hkl, ...), coverage
    iz0: np.ndarray                 # first frame index (0-based) of the box
    dz: np.ndarray                  # phi bins of the box (odd)
    fb: np.ndarray                  # frames per phi bin
    Dz: np.ndarray                  # depth bucket (>= dz): shoebox depth as stored
    bx: np.ndarray                  # box side (pixels or super-pixels)
    pxs: np.ndarray                 # super-pixel side
    ix0: np.ndarray                 # box origin in the reflection's own (super-)pixel units
    iy0: np.ndarray
    region: np.ndarray
    has_partner: np.ndarray
    partner: np.ndarray             # index of the nearest neighbour (the partner when has_partner)
    nb: dict                        # neighbour ellipsoids x, y, z, sx, sz: (n, K) float32
    overlap: np.ndarray
    nreg: int
    box: int
    blocks_refl: list               # rows of each block, in block-row order (stable by block)
    need_lo: list                   # first / last frame index each block needs
    need_hi: list
    zstart: np.ndarray
    zend: np.ndarray
    info: dict = field(default_factory=dict)
    dev: dict = field(default_factory=dict)      # device copies of the per-row columns (torch tensors)

    @property
    def nb_columns(self):
        return self.nb.columns if isinstance(self.nb, LazyHost) else int(self.nb["x"].shape[1])

    @property
    def n(self):
        return int(self.refl["x"].size)


class LazyHost(dict):
    """Host copies of device columns, made on first access (the integration itself reads them from the device)."""

    def __init__(self, dev, columns):
        super().__init__()
        self._dev = dev
        self.columns = columns

    def __missing__(self, k):
        v = self._dev[k].cpu().numpy()
        self[k] = v
        return v

    def items(self):
        return [(k, self[k]) for k in self._dev]

    def keys(self):
        return self._dev.keys()


def _segments(g):
    f = getattr(g, "segment_list", None) or getattr(g, "panel_list")
    return f()


def plan_detector(g, device="cuda"):
    """XiPlanDetector of a geometry: float64 panel records (`xpg/detector.py:79-90` maps and the per-panel constants
    of `xpg/geometry.py:269-310`, each computed with the reference's numpy expression) and the lab-map constants.
    Returns (struct, keep-alive tensors)."""
    P0, Bx, By = (np.asarray(a, np.float64).reshape(-1, 3) for a in g.panels())
    segs = _segments(g)
    K = P0.shape[0]
    rec = np.zeros((K, N.XI_PANEL_F64))
    for k in range(K):
        n = np.cross(Bx[k], By[k])
        u1, u2 = Bx[k] / g.qx, By[k] / g.qy
        rec[k, 0:3], rec[k, 3:6], rec[k, 6:9], rec[k, 9:12] = P0[k], Bx[k], By[k], n
        rec[k, 12:15], rec[k, 15:18], rec[k, 18:21] = u1, u2, np.cross(u1, u2)
        rec[k, 21], rec[k, 22], rec[k, 23] = P0[k] @ n, Bx[k] @ Bx[k], By[k] @ By[k]
        s = segs[min(k, len(segs) - 1)]
        rec[k, 24:28] = (s.x1, s.x2, s.y1, s.y2)
    d = N.XiPlanDetector()
    d.n_panels = K
    keep = {}
    if K <= N.XI_PANELS_INLINE:                 # carried in the kernel argument: no device copy
        d.panel_inline[:K * N.XI_PANEL_F64] = [float(v) for v in rec.reshape(-1)]
        d.panels = None
    else:
        keep["panels"] = h2d(rec, None, device)
        d.panels = N.ptr(keep["panels"])
    if getattr(g, "segmented", False):
        m = np.asarray(g.segmap(), np.int16)
        keep["segmap"] = torch.as_tensor(m).to(device)
        d.segmented, d.segmap = 1, N.ptr(keep["segmap"])
        d.seg_ny, d.seg_nx = m.shape
    geo = getattr(g, "geo_corr", None)
    if geo is not None:
        keep["gx"] = torch.as_tensor(np.asarray(geo[0], np.float64)).to(device)
        keep["gy"] = torch.as_tensor(np.asarray(geo[1], np.float64)).to(device)
        d.geo_x, d.geo_y = N.ptr(keep["gx"]), N.ptr(keep["gy"])
        d.geo_ny, d.geo_nx = keep["gx"].shape
    if g.has_parallax:
        d.parallax, d.tsens, d.mu = 1, float(g.sensor_thickness), float(g.mu)
    d.orgx, d.orgy, d.qx, d.qy, d.distance = (float(v) for v in (g.orgx, g.orgy, g.qx, g.qy, g.distance))
    e0 = np.asarray(g.beam, np.float64)
    pn = np.asarray(g.polarization_normal, np.float64)
    nvec = pn - np.dot(pn, e0) * e0
    nvec = nvec / np.linalg.norm(nvec)
    emain = np.cross(nvec, e0)
    for name, v in (("ed1", g.ed1), ("ed2", g.ed2), ("ed3", g.ed3), ("beam", e0), ("pol_n", nvec),
                    ("pol_main", emain)):
        getattr(d, name)[:] = [float(c) for c in np.asarray(v, np.float64)]
    d.pol_f = float(g.polarization_fraction)
    d.nx, d.ny = float(g.nx), float(g.ny)
    return d, keep


_CENTRING = {"P": ord("P"), "C": ord("C"), "A": ord("A"), "B": ord("B"), "I": ord("I"), "F": ord("F"),
             "R": ord("R")}


def _predict_struct(exp, g0, za, zb, dmin, dmax, z_lo, z_hi, minimum_zeta, block, lattice, allowed, device):
    """XiPredict of one phi block (`xpg/integrate.py:101-122`, `xpg/geometry.py:468-545`)."""
    g = exp.geom
    A = np.asarray(exp.crystal.Astar, np.float64)
    P = N.XiPredict()
    P.astar[:] = [float(v) for v in A.reshape(-1)]
    keep = None
    sym = str(exp.crystal.space_group).strip().upper()[:1]
    if allowed is centring_allowed:
        real = np.linalg.inv(A)
        P.hmax[:] = [int(np.ceil(np.linalg.norm(real[i]) / dmin)) for i in range(3)]
        P.q2_max, P.q2_min = 1.0 / dmin ** 2, 1.0 / dmax ** 2
        P.centring = _CENTRING.get(sym, ord("P"))
    else:                                   # a caller's own absence rule: its Miller-index list, in order
        hkl = generate_hkl(A, dmin, dmax)
        hkl = np.ascontiguousarray(hkl[allowed(hkl, exp.crystal.space_group)], np.int32)
        keep = h2d(hkl, None, device)
        P.hkl, P.n_hkl = N.ptr(keep), int(hkl.shape[0])
    axis = np.asarray(g.axis, np.float64)
    k = unit(axis)
    K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    P.axis[:] = [float(v) for v in axis]
    P.rot_K[:] = [float(v) for v in K.reshape(-1)]
    P.rot_kk[:] = [float(v) for v in np.outer(k, k).reshape(-1)]
    P.s0[:] = [float(v) for v in np.asarray(g.s0, np.float64)]
    lo, hi = sorted(g.z_to_phi(np.array((za, zb), float)))
    P.phi_lo, P.phi_hi = float(lo), float(hi)
    P.phi0, P.osc, P.z_shift = float(g.phi0), float(g.osc), float(g.starting_frame - 1)
    P.deg, P.rad = 180.0 / math.pi, math.pi / 180.0
    P.acc_s0[:] = [float(v) for v in np.asarray(g0.s0, np.float64)]
    P.acc_axis[:] = [float(v) for v in np.asarray(g0.axis, np.float64)]
    P.min_zeta = float(minimum_zeta)
    P.x_hi, P.y_hi = g0.nx + 0.5, g0.ny + 0.5
    P.z_lo, P.z_hi = float(z_lo), float(z_hi)
    P.block, P.lattice = int(block), int(lattice)
    return P, keep


PRED_F64 = ("phi", "x", "y", "z", "zeta", "polarization", "zeta_k")
BOX_I32 = ("iz0", "dz", "fb", "Dz", "bx", "pxs", "ix0", "iy0", "region", "zstart", "zend")


def _host_cols(cols):
    """Device columns -> host numpy arrays: the columns of one dtype and size go in one stacked copy through pinned
    memory (each column a contiguous row of it) instead of one synchronising copy each."""
    groups = {}
    for k, v in cols.items():
        groups.setdefault((v.dtype, v.numel()), []).append(k)
    out = {}
    for ks in groups.values():
        st = d2h(torch.stack([cols[k].reshape(-1) for k in ks]))
        for i, k in enumerate(ks):
            out[k] = st[i].reshape(tuple(cols[k].shape))
    return out


def _columns(n, names, dtype, device, width=None):
    return {k: torch.empty((n,) if not width or k not in width else (n, width[k]), dtype=dtype, device=device)
            for k in names}


def predict_device(exp_blocks, block_edges, dmin, dmax, z_lo, z_hi, minimum_zeta=0.05, lattice_of=None,
                   allowed=centring_allowed, device="cuda"):
    """Device predictions of every phi block (`xpg/integrate.py:101-122`): dict of torch columns in the reference's
    row order."""
    lib = N.load()
    st = N.stream_handle()
    g0 = exp_blocks[0].geom
    n_edges = len(block_edges) - 1
    det_cache = {}
    jobs = []
    for b, exp in enumerate(exp_blocks):
        za, zb = block_edges[b % n_edges], block_edges[b % n_edges + 1]
        P, keep = _predict_struct(exp, g0, za, zb, dmin, dmax, z_lo, z_hi, minimum_zeta, b,
                                  0 if lattice_of is None else lattice_of[b], allowed, device)
        key = id(exp.geom)
        if key not in det_cache:
            det_cache[key] = plan_detector(exp.geom, device)
        ws = torch.empty(max(int(lib.xi_predict_workspace(C.byref(P))), 1), dtype=torch.uint8, device=device)
        n = C.c_int64(0)
        with TIMER.span("plan", 2):             # k_predict_count, k_total (plus the library scan)
            N.check(lib.xi_predict_count(C.byref(P), C.byref(det_cache[key][0]), N.ptr(ws), ws.numel(), C.byref(n),
                                         st), "xi_predict_count")
        jobs.append((P, keep, key, ws, int(n.value)))
    total = sum(j[4] for j in jobs)
    cols = _columns(total, PRED_F64, torch.float64, device)
    cols["S"] = torch.empty((total, 3), dtype=torch.float64, device=device)
    cols["hkl"] = torch.empty((total, 3), dtype=torch.int32, device=device)
    cols["block"] = torch.empty(total, dtype=torch.int32, device=device)
    cols["lattice"] = torch.empty(total, dtype=torch.int32, device=device)
    o = 0
    for P, keep, key, ws, n in jobs:
        if n:
            out = N.XiPredictOut()
            for k, v in cols.items():
                setattr(out, k, N.ptr(v[o:o + n]))
            with TIMER.span("plan"):
                N.check(lib.xi_predict_write(C.byref(P), C.byref(det_cache[key][0]), N.ptr(ws), ws.numel(),
                                             C.byref(out), n, st), "xi_predict_write")
        o += n
    return cols


def _select(cols, keep_t):
    return {k: v[keep_t] for k, v in cols.items()}


def plan_integration(exp_blocks, block_edges, model, dmin, dmax=1e9, frames=(1, 1), minimum_zeta=0.05,
                     n_regions_xy=3, adaptive=True, deconvolve_overlaps=True, lattice_of=None, foreign_spots=None,
                     n_foreign=4, allowed=centring_allowed, device="cuda"):
    """Predictions and shoebox plan of a sweep on the device (`xpg/integrate.py:222-370`)."""
    N.require_cuda()
    lib = N.load()
    st = N.stream_handle()
    g0 = exp_blocks[0].geom
    f_first, f_last = frames
    z_lo, z_hi = f_first - 1.0, float(f_last)
    pred = predict_device(exp_blocks, block_edges, dmin, dmax, z_lo, z_hi, minimum_zeta, lattice_of, allowed, device)
    n_pred = int(pred["x"].shape[0])
    widen = 1.3 if adaptive else 1.0
    box = (IntegrationModel(model.sigma_d * widen, model.sigma_m).box(g0) if not model.box_xy else model.box_xy)
    # shoebox rules (`xpg/integrate.py:233-291`, `:316-318`)
    det0, keep0 = plan_detector(g0, device)
    B = N.XiBoxRules()
    B.n = n_pred
    for k in ("x", "y", "z", "zeta_k"):
        setattr(B, k, N.ptr(pred[k]))
    B.sigma_m = float(model.sigma_m)
    B.abs_osc = float(abs(g0.osc))
    B.osc2_12 = float((g0.osc ** 2) / 12.0)
    B.rsd_box = float(np.radians(model.sigma_d * widen))
    B.rsd = float(np.radians(model.sigma_d))
    B.qmin = float(min(g0.qx, g0.qy))
    B.box = int(box)
    B.box_fixed = 1 if model.box_xy else 0
    xyb = [b_ for b_ in XY_BUCKETS if b_ < box] + [box]
    B.n_xyb = len(xyb)
    B.xyb[:len(xyb)] = [int(v) for v in xyb]
    B.f_first, B.f_last = int(f_first), int(f_last)
    B.n_regions_xy = int(n_regions_xy)
    bcols = _columns(n_pred, BOX_I32, torch.int32, device)
    bcols["flags"] = torch.empty(n_pred, dtype=torch.uint8, device=device)
    bcols["coverage"] = torch.empty(n_pred, dtype=torch.float32, device=device)
    bcols["sx_px"] = torch.empty(n_pred, dtype=torch.float64, device=device)
    bcols["sz_f"] = torch.empty(n_pred, dtype=torch.float64, device=device)
    O = N.XiBoxOut()
    for k, v in bcols.items():
        setattr(O, k, N.ptr(v))
    with TIMER.span("plan"):
        N.check(lib.xi_plan_boxes(C.byref(B), C.byref(det0), C.byref(O), st), "xi_plan_boxes")
    flags = bcols.pop("flags")
    fl = flags.cpu().numpy()
    info = dict(n_predicted=n_pred, n_wide=int((fl & 1).sum()), n_trunc=int(((fl & 2) > 0).sum()), box=box)
    if not (fl & 4).all():                  # rows without a depth bucket leave the plan
        keep_t = h2d((fl & 4) > 0, None, device)
        pred, bcols = _select(pred, keep_t), _select(bcols, keep_t)
    n = int(pred["x"].shape[0])
    # neighbour lists on the mean scales (`xpg/integrate.py:164-172`, `:287-303`)
    sx_h = bcols["sx_px"].cpu().numpy()
    sz_h = bcols["sz_f"].cpu().numpy()
    K = K_NEIGHBOURS
    nbj = torch.zeros((n, K), dtype=torch.int32, device=device)
    nbd = torch.full((n, K), float("inf"), dtype=torch.float64, device=device)
    sxm = szm = 1.0
    if n:
        sxm, szm = float(sx_h.mean()), float(sz_h.mean())
        q = N.XiKnn()
        q.n, q.x, q.y, q.z = n, N.ptr(pred["x"]), N.ptr(pred["y"]), N.ptr(pred["z"])
        q.sx, q.sz = sxm, szm
        q.lo[:] = [0.5 / sxm, 0.5 / sxm, z_lo / szm]
        q.hi[:] = [(g0.nx + 0.5) / sxm, (g0.ny + 0.5) / sxm, z_hi / szm]
        q.radius, q.k = 4.0 * N_FG, K
        ws = torch.empty(max(int(lib.xi_knn_workspace(C.byref(q))), 1), dtype=torch.uint8, device=device)
        with TIMER.span("plan", 3):             # k_knn_bin, k_knn_scatter, k_knn_query (plus the library scan)
            N.check(lib.xi_knn(C.byref(q), N.ptr(ws), ws.numel(), N.ptr(nbj), N.ptr(nbd), st), "xi_knn")
    has = torch.isfinite(nbd)
    jl = nbj.long()
    has_partner = (has[:, 0] & (nbd[:, 0] < 2.0)) if (deconvolve_overlaps and n) else torch.zeros(n, dtype=torch.bool,
                                                                                                   device=device)
    f32 = lambda t: t.to(torch.float32)
    nb = dict(x=f32(torch.where(has, pred["x"][jl], -1e6)), y=f32(torch.where(has, pred["y"][jl], -1e6)),
              z=f32(torch.where(has, pred["z"][jl], -1e6)), sx=f32(torch.where(has, bcols["sx_px"][jl], 1.0)),
              sz=f32(torch.where(has, bcols["sz_f"][jl], 1.0)))
    # host copies
    hc = _host_cols(dict(pred, **{"box_" + k: bcols[k].long() for k in BOX_I32}, coverage=bcols["coverage"],
                         has_partner=has_partner, partner=nbj[:, 0].contiguous()))
    refl = {k: hc[k] for k in pred}
    h = {k: hc["box_" + k] for k in BOX_I32}
    refl["coverage"] = hc["coverage"]
    nbh = LazyHost(nb, K)
    hp = hc["has_partner"]
    partner = hc["partner"].astype(np.int64) if n else np.zeros(0, np.int64)
    if foreign_spots is not None and len(foreign_spots[0]) and n:
        nbh = {k: nbh[k] for k in ("x", "y", "z", "sx", "sz")}
        _add_foreign(nbh, refl, foreign_spots, n_foreign, sxm, szm)
    blk = refl["block"]
    nblocks = len(exp_blocks)
    if (blk[1:] >= blk[:-1]).all():        # predictions leave the planner in block order: ranges of rows
        bounds = np.searchsorted(blk, np.arange(nblocks + 1), side="left")
        blocks_refl = [np.arange(bounds[b], bounds[b + 1], dtype=np.int64) for b in range(nblocks)]
    else:
        order = np.argsort(blk, kind="stable")
        blocks_refl = [order[blk[order] == b] for b in range(nblocks)]
    zstart, zend = h["zstart"], h["zend"]
    need_lo = [int(zstart[r].min()) if r.size else 10 ** 9 for r in blocks_refl]
    need_hi = [int(zend[r].max()) if r.size else -1 for r in blocks_refl]
    dev = dict(pred, **bcols, nbj=nbj, nbd=nbd, has_partner=has_partner, **{"nb" + k: v for k, v in nb.items()})
    return Plan(refl=refl, iz0=h["iz0"], dz=h["dz"], fb=h["fb"], Dz=h["Dz"], bx=h["bx"], pxs=h["pxs"], ix0=h["ix0"],
                iy0=h["iy0"], region=h["region"].astype(np.int32), has_partner=hp, partner=partner, nb=nbh,
                overlap=hp.copy(), nreg=n_regions_xy * n_regions_xy, box=box, blocks_refl=blocks_refl,
                need_lo=need_lo, need_hi=need_hi, zstart=zstart, zend=zend, info=info, dev=dev)


def _add_foreign(nb, refl, foreign_spots, n_foreign, sxm, szm):
    """Neighbour columns of spots from other lattices or foreign sources (`xpg/integrate.py:304-315`): the
    n_foreign nearest spots within 4 N_FG but beyond 2.5 / N_FG, as small ellipsoids. A host search: the list is an
    optional input, usually short."""
    from scipy.spatial import cKDTree
    fx, fy, fz = (np.asarray(a, float) for a in foreign_spots)
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
