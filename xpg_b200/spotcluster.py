"""Clustering of strong pixels into spots (the second half of XPG's spot finding, `xpg/spotcluster.py:49-375`), on
the host: numpy / scipy, as in XPG, over the strong pixels the device classifier (`spotfind.make_finder`) leaves
(~0.03% of the pixels).

`cluster_spots` is the one-pass form: every strong pixel of a run at once, the spots XPG's accumulator gives when all
of them are added before one flush. Steps, each with XPG's rules:
* components: pixels within `cluster_radius` in-plane (Chebyshev) on the same or an adjacent frame are connected;
  components numbered by their first pixel in input order;
* splitting (`:87-238`): a pixel is a peak when its net value (value - background) is significant (> 3 sqrt(max(bg,
  1))) and not below any of its 26 neighbours present (ties: the pixel wins against neighbours at offsets below it
  in (dz, dy, dx) order); in a cluster with two or more peaks, peaks are taken by decreasing net value and kept when
  at least `min_sep_xy` px in-plane from every kept one and separated from each by a dip (the lowest strong pixel
  within 0.75 px of the segment between them, or background where the segment leaves the strong set, below the
  peak by more than 3 sqrt(max(value, 1))); in a huge cluster only kept peaks within 12 px are tested, over the pixels
  near the segment; the cluster's pixels go to the nearest kept peak (frames weighted 1.5);
* spot properties (`:329-375`): background-subtracted centroids and intensity, pixel count, frame range; spots are
  dropped outside [min_pix, max_pix] pixels, with no signal, or whose brightest pixel lies more than
  `max_centroid_dist` px from the centroid.
"""
from __future__ import annotations

import numpy as np
from scipy.sparse import coo_matrix
from scipy.sparse.csgraph import connected_components
from scipy.spatial import cKDTree

PIX0 = 1.0                     # coordinate of the centre of array element 0 (XPG's pixel convention)
NSIG = 3.0
MIN_SEP_XY = 2.0
PATH_HALF_WIDTH = 0.75         # pixels within this distance of a peak-to-peak segment lie on it
Z_WEIGHT = 1.5                 # frames against pixels when pixels go to their nearest peak
HUGE_PIXELS, HUGE_PEAKS = 20000, 200
NEAR_PEAKS = 12.0              # huge clusters: kept peaks farther than this (3D, px / frames) are separate


def _neighbour_offsets(r):
    """Offsets (dz, dy, dx) linking a pixel to the pixels after it: same frame within r (the half of the square after
    the pixel in row-major order), next frame within r."""
    same = [(0, dy, dx) for dy in range(0, r + 1) for dx in range(-r, r + 1) if dy > 0 or dx > 0]
    return same + [(1, dy, dx) for dy in range(-r, r + 1) for dx in range(-r, r + 1)]


def _sorted_lookup(key, x, y, nx, ny, offsets):
    """For every offset, the pairs (pixel, neighbour) present in the set; key: the pixels' linear voxel indices."""
    order = np.argsort(key)
    ks = key[order]
    n = key.size
    for dz, dy, dx in offsets:
        tgt = ks + (dz * ny + dy) * nx + dx
        pos = np.minimum(np.searchsorted(ks, tgt), n - 1)
        xs, ys = x[order], y[order]
        inside = (xs + dx >= 0) & (xs + dx < nx) & (ys + dy >= 0) & (ys + dy < ny)
        found = inside & (ks[pos] == tgt)
        yield (dz, dy, dx), order, pos, found


def components(z, y, x, nx, ny, radius=1):
    """Connected-component labels of the pixels (numbered by first pixel in input order) and their count."""
    n = z.size
    if n == 0:
        return np.zeros(0, np.int64), 0
    key = (z.astype(np.int64) * ny + y) * nx + x
    a, b = [], []
    for _, order, pos, found in _sorted_lookup(key, x, y, nx, ny, _neighbour_offsets(radius)):
        a.append(order[found])
        b.append(order[pos[found]])
    a, b = np.concatenate(a), np.concatenate(b)
    nc, lab = connected_components(coo_matrix((np.ones(a.size, np.int8), (a, b)), shape=(n, n)), directed=False)
    return lab.astype(np.int64), int(nc)


def _peaks(z, y, x, net, b, nx, ny):
    key = (z.astype(np.int64) * ny + y) * nx + x
    offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dz, dy, dx) != (0, 0, 0)]
    peak = None
    for off, order, pos, found in _sorted_lookup(key, x, y, nx, ny, offs):
        mine = net[order]
        if peak is None:
            peak = mine > NSIG * np.sqrt(np.maximum(b[order], 1.0))
        other = np.where(found, net[order][pos], -np.inf)
        peak &= (mine > other) | ((mine == other) & (off > (0, 0, 0)))
    out = np.empty(z.size, bool)
    out[np.argsort(key)] = peak
    return out


def _dip_below(q, r_list, px, cnet, net, thr, coords):
    """Every r in r_list is separated from peak q by a significant dip (over the given candidate pixels px)."""
    x, y, z = coords
    for r in r_list:
        a0, a1, a2 = float(x[r]), float(y[r]), float(z[r])
        d0, d1, d2 = x[q] - a0, y[q] - a1, z[q] - a2
        L2 = d0 * d0 + d1 * d1 + d2 * d2
        c0, c1, c2 = px[:, 0] - a0, px[:, 1] - a1, px[:, 2] - a2
        t = np.clip((c0 * d0 + c1 * d1 + c2 * d2) / L2, 0, 1)
        dist = np.sqrt((c0 - t * d0) ** 2 + (c1 - t * d1) ** 2 + (c2 - t * d2) ** 2)
        on = (dist <= PATH_HALF_WIDTH) & (t > 0) & (t < 1)
        steps = int(np.ceil(np.sqrt(L2))) - 1
        saddle = cnet[on].min() if (on.any() and on.sum() >= steps) else np.float32(0.0)
        if not net[q] - saddle > thr[q]:
            return False
    return True


def split_merged(z, y, x, v, b, lab, nx, ny):
    """Labels after splitting clusters of touching spots at their separated peaks: label * stride + 1 + peak rank in
    a split cluster, label * stride elsewhere (stride 1 when nothing splits, else at least 4096)."""
    n = z.size
    if n == 0:
        return lab
    net = v - b
    pk = np.flatnonzero(_peaks(z, y, x, net, b, nx, ny))
    if pk.size == 0:
        return lab
    multi = np.flatnonzero(np.bincount(lab[pk], minlength=int(lab.max()) + 1) >= 2)
    if multi.size == 0:
        return lab
    thr = NSIG * np.sqrt(np.maximum(v, np.float32(1.0)))
    sub = np.zeros(n, np.int64)
    most = 0
    by_lab = np.argsort(lab, kind="stable")
    lo, hi = np.searchsorted(lab[by_lab], multi), np.searchsorted(lab[by_lab], multi, "right")
    pk = pk[np.argsort(lab[pk], kind="stable")]
    plo, phi_ = np.searchsorted(lab[pk], multi), np.searchsorted(lab[pk], multi, "right")
    for i in range(multi.size):
        pix = by_lab[lo[i]:hi[i]]
        pks = pk[plo[i]:phi_[i]]
        pks = pks[np.argsort(-net[pks], kind="stable")]
        P = np.c_[x[pix], y[pix], z[pix]].astype(float)
        cnet = net[pix]
        huge = pix.size > HUGE_PIXELS or pks.size > HUGE_PEAKS
        kept = [int(pks[0])]
        if huge:
            tree = cKDTree(P)
            cell = int(np.ceil(max(4.0 * MIN_SEP_XY, NEAR_PEAKS)))
            grid = {}
            m = int(np.ceil(MIN_SEP_XY))
            disc = [(dy, dx) for dy in range(-m, m + 1) for dx in range(-m, m + 1) if np.hypot(dy, dx) < MIN_SEP_XY]
            near_peak = set()

            def keep(q):
                for dy, dx in disc:
                    near_peak.add((int(y[q]) + dy, int(x[q]) + dx))
                grid.setdefault((int(x[q]) // cell, int(y[q]) // cell), []).append(q)

            def separated(q):
                if (int(y[q]), int(x[q])) in near_peak:
                    return False
                cx, cy = int(x[q]) // cell, int(y[q]) // cell
                rs = sorted(r for gx in (cx - 1, cx, cx + 1) for gy in (cy - 1, cy, cy + 1) for r in grid.get((gx, gy), ()))
                for r in rs:
                    D = np.sqrt(np.hypot(x[q] - x[r], y[q] - y[r]) ** 2 + float(z[q] - z[r]) ** 2)
                    if D > max(4.0 * MIN_SEP_XY, NEAR_PEAKS):
                        continue
                    a0, a1, a2 = float(x[r]), float(y[r]), float(z[r])
                    d0, d1, d2 = x[q] - a0, y[q] - a1, z[q] - a2
                    ball = tree.query_ball_point([(x[q] + a0) / 2, (y[q] + a1) / 2, (z[q] + a2) / 2],
                                                 np.sqrt(d0 * d0 + d1 * d1 + d2 * d2) / 2 + 1.0)
                    if not ball:
                        continue
                    ball = np.asarray(ball)
                    if not _dip_below(q, [r], P[ball], cnet[ball], net, thr, (x, y, z)):
                        return False
                return True

            keep(kept[0])
        else:
            def separated(q):
                ks = np.asarray(kept)
                if not (np.hypot(x[q] - x[ks], y[q] - y[ks]) >= MIN_SEP_XY).all():
                    return False
                return _dip_below(q, kept, P, cnet, net, thr, (x, y, z))

        for q in pks[1:]:
            q = int(q)
            if separated(q):
                kept.append(q)
                if huge:
                    keep(q)
        if len(kept) < 2:
            continue
        kp = np.asarray(kept)
        _, nearest = cKDTree(np.c_[x[kp], y[kp], z[kp] * Z_WEIGHT]).query(np.c_[x[pix], y[pix], z[pix] * Z_WEIGHT])
        sub[pix] = 1 + nearest
        most = max(most, len(kept))
    return lab.astype(np.int64) * max(4096, most + 1) + sub


def spot_properties(z, y, x, v, b, lab, min_pix, max_pix, max_centroid_dist, parent_last=None):
    """Per spot (in label order): centroid x, y, z (pixel and frame centres), intensity, pixel count, first frame,
    last frame + 1; spots outside the pixel-count range, without signal or off-centre dropped. parent_last: per
    pixel, the last frame of its unsplit cluster, returned per spot as `parent_last`."""
    _, first, lab = np.unique(lab, return_index=True, return_inverse=True)
    nc = int(lab.max()) + 1 if lab.size else 0
    w = np.maximum(v - b, 0.0).astype(np.float64)
    npix = np.bincount(lab, minlength=nc)
    sw = np.bincount(lab, w, nc)
    den = np.where(sw > 0, sw, 1.0)
    cx = np.bincount(lab, w * (x + PIX0), nc) / den
    cy = np.bincount(lab, w * (y + PIX0), nc) / den
    cz = np.bincount(lab, w * (z + 0.5), nc) / den
    zmin = np.full(nc, 1 << 30)
    zmax = np.full(nc, -1)
    np.minimum.at(zmin, lab, z)
    np.maximum.at(zmax, lab, z)
    srt = np.lexsort((v, lab))                 # by spot, then value: each spot's brightest pixel last
    brightest = srt[np.r_[np.flatnonzero(np.diff(lab[srt])), lab.size - 1]] if lab.size else srt
    off = np.hypot(x[brightest] + PIX0 - cx, y[brightest] + PIX0 - cy)
    ok = (npix >= min_pix) & (npix <= max_pix) & (sw > 0) & (off <= max_centroid_dist)
    out = dict(x=cx[ok], y=cy[ok], z=cz[ok], intensity=sw[ok], npix=npix[ok], zmin=zmin[ok].astype(float),
               zmax=zmax[ok] + 1.0)
    if parent_last is not None:
        out["parent_last"] = np.asarray(parent_last)[first][ok]
    return out


def cluster_spots(z, y, x, v, b, nx, ny, min_pix, max_pix, max_centroid_dist=3.0, cluster_radius=2,
                  with_parents=False):
    """Spots of strong pixels (frame index z, row y, column x, value v, local background b, in frame-major, row-major
    order), all at once; with_parents adds each spot's unsplit cluster's last frame (`parent_last`)."""
    z, y, x = (np.asarray(a, np.int32) for a in (z, y, x))
    v, b = np.asarray(v, np.float32), np.asarray(b, np.float32)
    if z.size == 0:
        e = np.zeros(0)
        out = dict(x=e, y=e, z=e, intensity=e, npix=e.astype(int), zmin=e, zmax=e)
        if with_parents:
            out["parent_last"] = e.astype(np.int64)
        return out
    lab, nc = components(z, y, x, nx, ny, cluster_radius)
    last = None
    if with_parents:
        zc = np.full(nc, -1, np.int64)
        np.maximum.at(zc, lab, z)
        last = zc[lab]
    lab = split_merged(z, y, x, v, b, lab, nx, ny)
    return spot_properties(z, y, x, v, b, lab, min_pix, max_pix, max_centroid_dist, last)


def flush_thresholds(batches):
    """The flushes of XPG's streaming clustering over frame batches (`xpg/spotcluster.py:378-402`): after each batch,
    clusters ending before its last frame close; at a gap in the frame numbers every open cluster closes; the last
    flush closes the rest. Returns the thresholds (0-based frames, non-decreasing): a cluster closes at the first
    flush whose threshold exceeds its last frame."""
    c, prev = [], None
    for fr in batches:
        for f in fr:
            if prev is not None and f != prev + 1:
                c.append(prev)
            prev = f
        c.append(prev - 1)
    c.append(np.iinfo(np.int64).max)
    return np.array(c, np.int64)


def streaming_order(spots, batches):
    """The order XPG's streaming clustering emits the spots of `cluster_spots(..., with_parents=True)` in: by the
    flush that closes their cluster, then as the one pass orders them (clusters by first pixel, split spots by peak)."""
    flush = np.searchsorted(flush_thresholds(batches), spots["parent_last"], side="right")
    return np.argsort(flush, kind="stable")
