"""Device-memory planning of an integration run: the shoebox arenas and per-row buffers of the phi blocks open at once
must fit the device.

XPG keeps its shoebox buffers in host memory and plans for it (`_integrate_budget`, `_plan_passes`, `_split_blocks`,
xpg/shoebox.py:118-196, used at xpg/integrate.py:592-626): a block's buffers are held from the first frame any of its
boxes needs until its last reflection is complete, and when the peak over the frames does not fit, each phi block is
integrated in k parts of consecutive phi (about equal shoebox bytes each; the fewest parts that fit, at most 8), each
part with its own learnt profiles and widths. Here the buffers live in HBM, so the same accounting runs against the
device's memory; the parts keep the reference's rule (rows of a block ordered by z, cut at equal cumulative bytes).
"""
from __future__ import annotations

import os
from dataclasses import replace

import numpy as np

BLOCK_PARTS_MAX = 8          # parts per phi block at most (xpg/integrate.py:55)
DEVICE_FRACTION = 0.95       # share of the device memory free at the start that the run's buffers may use
WIDE_SPANS = 4.0             # rows deeper in phi than this many median spans: a part of their own (frames read once)


def _bytes_of(Dz, bx, binned):
    Dz = np.asarray(Dz, np.int64)
    bx = np.asarray(bx, np.int64)
    arena = 4 * ((Dz * bx * bx + 3) & ~3)
    return arena + arena // 20 + np.where(binned, 4 * Dz, 0) + 17 * bx * bx + 4 * Dz + 400     # + the pool's 5%


_TABLE = _bytes_of(*np.meshgrid(np.arange(128), np.arange(128), np.arange(2), indexing="ij")).reshape(-1)


def row_bytes(plan):
    """Device bytes of every row while its block is open: the shoebox (value + 3 floats, rows on 16 bytes, and the
    buffer pool's 5% slack), bin counters of binned rows, the per-pixel pass-1 tables (img2, J, u1, u2,
    all_valid2), per-frame fz, per-row scalars of both passes. Depths and sides come from short bucket lists, so a
    table over (depth, side, binned) below 128 answers every row with one gather (millions of rows per plan)."""
    Dz = np.asarray(plan.Dz).astype(np.int32, copy=False)
    bx = np.asarray(plan.bx).astype(np.int32, copy=False)
    binned = np.asarray(plan.fb) > 1
    if Dz.size:
        code = Dz << 8
        code |= bx << 1
        lo, hi = int(code.min()), int(code.max())
        if 0 <= lo and hi < (128 << 8) and 0 <= int(bx.min()) and int(bx.max()) < 128:
            code |= binned
            return _TABLE[code]
    return _bytes_of(Dz, bx, binned)


def budget(device="cuda"):
    """Bytes the run's shoebox buffers may use: XPG_INTEGRATE_MEM_GB (the reference's knob for the same buffers), else
    DEVICE_FRACTION of the device memory free now (the caching allocator's free blocks and the buffer pool's kept
    buffers counted as free)."""
    gb = os.environ.get("XPG_INTEGRATE_MEM_GB")
    if gb:
        return float(gb) * 2 ** 30
    import torch
    dev = torch.device(device)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    from .device import POOL
    kept = sum(t.numel() * t.element_size() for (d, _), ts in POOL.free.items() if d == dev.index for t in ts)
    free = (torch.cuda.mem_get_info(dev)[0] + torch.cuda.memory_reserved(dev) - torch.cuda.memory_allocated(dev)
            + kept)
    return DEVICE_FRACTION * free


def peak_bytes(blocks_refl, need_lo, need_hi, w_row, n_frames):
    """Largest sum over the frames of the bytes of the blocks open at that frame (block b open over frame indices
    need_lo[b]..need_hi[b]), and the largest single block."""
    d = np.zeros(n_frames + 2)
    big = 0.0
    for b, rows in enumerate(blocks_refl):
        if rows.size:
            w = float(w_row[rows].sum())
            d[int(np.clip(need_lo[b], 0, n_frames))] += w
            d[int(np.clip(need_hi[b] + 1, 0, n_frames + 1))] -= w
            big = max(big, w)
    return float(np.cumsum(d).max()), big


def _rows_sum(w, rows):
    """w summed over a block's rows (sorted, distinct plan rows: a slice when they are a range)."""
    if not rows.size:
        return 0.0
    a, e = int(rows[0]), int(rows[-1]) + 1
    return float(w[a:e].sum() if e - a == rows.size else w[rows].sum())


def peak_of(nbytes, lo, hi, n_frames):
    """Largest sum over the frames of `nbytes[i]` for the parts open at the frame (part i over frame indices
    lo[i]..hi[i])."""
    nbytes = np.asarray(nbytes, np.float64)
    if not nbytes.size:
        return 0.0
    d = np.zeros(n_frames + 2)
    np.add.at(d, np.clip(np.asarray(lo, np.int64), 0, n_frames), nbytes)
    np.add.at(d, np.clip(np.asarray(hi, np.int64) + 1, 0, n_frames + 1), -nbytes)
    return float(np.cumsum(d).max())


class _Cuts:
    """A split's parts without their row lists: per part its bytes, first and last frame, block, and where its rows
    lie in its block's z order (`rows()` makes the row lists of the chosen split only)."""

    def __init__(self):
        self.nbytes, self.lo, self.hi, self.parent, self.slices = [], [], [], [], []

    def add(self, nbytes, lo, hi, parent, sl):
        self.nbytes.append(nbytes)
        self.lo.append(int(lo))
        self.hi.append(int(hi))
        self.parent.append(parent)
        self.slices.append(sl)

    def peak(self, n_frames):
        return peak_of(self.nbytes, self.lo, self.hi, n_frames)

    def rows(self):
        return [np.sort(o[a:e]) for o, a, e in self.slices]


class _ZOrders:
    """Every block's rows (optionally a subset) in z order, with their cumulative bytes and frame bounds: sorted once,
    cut for every k."""

    def __init__(self, blocks_refl, z, w_row, zstart, zend, keep=None):
        self.items = []
        for b, rows in enumerate(blocks_refl):
            r = rows if keep is None else rows[keep[rows]]
            if not r.size:
                continue
            o = r[np.argsort(z[r], kind="stable")]
            c = np.concatenate([[0.0], np.cumsum(w_row[o], dtype=np.float64)])
            self.items.append((b, o, c, np.asarray(zstart)[o], np.asarray(zend)[o]))

    def subset(self, keep):
        """The same orders restricted to the rows where `keep` (a boolean per row) holds: no new sort."""
        out = _ZOrders.__new__(_ZOrders)
        out.items = []
        for b, o, c, zs, ze in self.items:
            m = keep[o]
            if not m.any():
                continue
            step = np.diff(c)[m]
            out.items.append((b, o[m], np.concatenate([[0.0], np.cumsum(step)]), zs[m], ze[m]))
        return out

    def cut(self, k, out=None):
        """Every block in k parts of consecutive z with about equal bytes (XPG's `_split_blocks` rule: cuts where the
        cumulative bytes pass k equal shares; empty parts dropped)."""
        out = out if out is not None else _Cuts()
        for b, o, c, zs, ze in self.items:
            cuts = np.searchsorted(c[1:], c[-1] * np.arange(1, k) / k, side="right")
            edges = np.unique(np.concatenate([[0], cuts, [o.size]]))
            a, e = edges[:-1], edges[1:]
            lo, hi = np.minimum.reduceat(zs, a), np.maximum.reduceat(ze, a)
            for i in range(a.size):
                out.add(float(c[e[i]] - c[a[i]]), lo[i], hi[i], b, (o, int(a[i]), int(e[i])))
        return out


def split_blocks(blocks_refl, z, w_row, k):
    """Every block's rows in k parts of consecutive z with about equal bytes (rows in index order within a part;
    empty parts dropped): (parts, the block of each part)."""
    n = int(max((int(r.max()) + 1 for r in blocks_refl if r.size), default=0))
    cuts = _ZOrders(blocks_refl, z, w_row, np.zeros(n, np.int64), np.zeros(n, np.int64)).cut(k)
    return cuts.rows(), cuts.parent


def fit(plan, exp_blocks, n_frames, wedge_bytes, limit, allow_passes=True):
    """The plan (and per-block experiments) whose open blocks fit `limit` bytes with the wedge buffers, in XPG's
    order (xpg/integrate.py:598-622): unchanged when one pass over the frames fits; else, when the frames can be read
    again (allow_passes), the whole blocks in several passes over the frames (`split_passes`); else every block split
    into the fewest parts of consecutive phi (2..8) that fit, each split with its own passes (allow_passes), or the
    split with the lowest peak when none fits and it is below the whole blocks'. Frames read once (no passes) and no
    such split fits: the rows far deeper in phi than the others in a part of their own (`split_wide`, info
    ["wide_apart"]). Returns (plan, exp_blocks, info); info["passes"]: the block lists of the passes when there are
    several; info["parts"]: parts per block of the consecutive-phi split."""
    w_row = row_bytes(plan)
    nb = [_rows_sum(w_row, r) for r in plan.blocks_refl]
    one = peak_of(nb, plan.need_lo, plan.need_hi, n_frames)
    info = dict(peak=one + wedge_bytes, one=one + wedge_bytes, parts=1, budget=limit)
    if limit is None or one + wedge_bytes <= limit:
        return plan, exp_blocks, info
    room = limit - wedge_bytes
    lat = plan.refl.get("lattice")

    def passes_of(nbytes, lo, hi, first_rows):
        if not allow_passes:
            return [], None
        lattice = [int(lat[r]) if lat is not None and r >= 0 else 0 for r in first_rows]
        return split_passes(nbytes, lo, hi, lattice, n_frames, room)

    base, base_pk = passes_of(nb, plan.need_lo, plan.need_hi, [int(r[0]) if r.size else -1 for r in plan.blocks_refl])
    whole = base_pk if base_pk is not None else one
    if base_pk is not None and base_pk <= room:
        info.update(peak=base_pk + wedge_bytes, passes=base)
        return plan, exp_blocks, info
    zo = _ZOrders(plan.blocks_refl, plan.refl["z"], w_row, plan.zstart, plan.zend)
    best = None
    for k in range(2, BLOCK_PARTS_MAX + 1):
        cuts = zo.cut(k)
        passes, pk = passes_of(cuts.nbytes, cuts.lo, cuts.hi, [int(o[a]) for o, a, _ in cuts.slices])
        if pk is None:
            pk = cuts.peak(n_frames)
        if best is None or pk < best[0]:
            best = (pk, k, cuts, passes, False)
        if pk <= room:
            break
    if not allow_passes and best[0] > room:
        # frames read once and no split by XPG's rule fits: a few rows far deeper in phi than a part (binned, near
        # the rotation axis) keep every part of their block open; those rows go in a part of their own
        wide = wide_rows(plan.blocks_refl, plan.zstart, plan.zend)
        zn, zw = zo.subset(~wide), zo.subset(wide)
        for k in range(2, BLOCK_PARTS_MAX + 1):
            cuts = _wide_cut(zn, zw, k)
            pk = cuts.peak(n_frames)
            if pk < best[0]:
                best = (pk, k, cuts, [], True)
            if pk <= room:
                break
    pk, k, cuts, passes, wide = best
    if pk < whole:
        lo, hi = list(cuts.lo), list(cuts.hi)
        plan = replace(plan, blocks_refl=cuts.rows(), need_lo=lo, need_hi=hi)
        exp_blocks = [exp_blocks[b] for b in cuts.parent]
        info.update(peak=pk + wedge_bytes, parts=k, parent=list(cuts.parent))
        if wide:
            info["wide_apart"] = True
        if len(passes) > 1:
            info["passes"] = passes
    elif base_pk is not None and base_pk < one:
        info.update(peak=base_pk + wedge_bytes, passes=base)
    return plan, exp_blocks, info


def wide_rows(blocks_refl, zstart, zend):
    """Rows whose frame span exceeds WIDE_SPANS times the median span of the plan's rows (a boolean per row)."""
    span = np.asarray(zend, np.int64) - np.asarray(zstart, np.int64) + 1
    nonempty = [r for r in blocks_refl if r.size]
    if not nonempty:
        return np.zeros(span.size, bool)
    return span > max(8.0, WIDE_SPANS * float(np.median(span[np.concatenate(nonempty)])))


def _wide_cut(z_narrow, z_wide, k):
    """Each block's other rows in k parts by XPG's rule, then its wide rows as one part (`split_wide`)."""
    narrow = z_narrow.cut(k)
    wide = z_wide.cut(1)
    out = _Cuts()
    by_block = {}
    for i, b in enumerate(wide.parent):
        by_block[b] = i
    blocks = sorted(set(narrow.parent) | set(wide.parent))
    for b in blocks:
        for i, pb in enumerate(narrow.parent):
            if pb == b:
                out.add(narrow.nbytes[i], narrow.lo[i], narrow.hi[i], b, narrow.slices[i])
        if b in by_block:
            i = by_block[b]
            out.add(wide.nbytes[i], wide.lo[i], wide.hi[i], b, wide.slices[i])
    return out


def split_wide(blocks_refl, z, zstart, zend, w_row, k):
    """Every block's rows whose frame span exceeds WIDE_SPANS times the median span in a part of their own (after the
    block's other parts), the other rows in k parts by XPG's rule (`split_blocks`): (parts, the block of each part).
    No counterpart in XPG, which can always read the frames again instead."""
    wide = wide_rows(blocks_refl, zstart, zend)
    cuts = _wide_cut(_ZOrders(blocks_refl, z, w_row, zstart, zend, keep=~wide),
                     _ZOrders(blocks_refl, z, w_row, zstart, zend, keep=wide), k)
    return cuts.rows(), cuts.parent


def split_passes(nbytes, need_lo, need_hi, lattice, n_frames, limit, max_passes=16):
    """Passes over the frames whose open blocks fit `limit` bytes, XPG's candidates in its order (`_plan_passes`,
    xpg/shoebox.py:134-183): one pass, then by lattice (blocks of other lattices cover the same frames), then within
    each lattice the blocks m apart in phi; the first that fits, else the fewest passes within 5% of the lowest peak.
    nbytes: each block's bytes (empty blocks, 0, take no pass). Returns (passes: block index lists in phi order, their
    peak)."""
    nbytes = np.asarray(nbytes, np.float64)
    lo_a, hi_a = np.asarray(need_lo, np.int64), np.asarray(need_hi, np.int64)
    order = sorted((b for b in range(nbytes.size) if nbytes[b] > 0), key=lambda b: lo_a[b])
    lat = [lattice[b] for b in order]
    lats = sorted(set(lat))
    rank, seen = [], {}
    for l_ in lat:
        rank.append(seen.get(l_, 0))
        seen[l_] = rank[-1] + 1
    cands = [[0] * len(order)]
    cands += [[lats.index(l_) % k for l_ in lat] for k in range(2, len(lats) + 1)]
    cands += [[lats.index(l_) * m + r % m for l_, r in zip(lat, rank)] for m in range(2, max_passes // len(lats) + 1)]
    tried = []
    for key in cands:
        passes = [[b for b, k_ in zip(order, key) if k_ == q] for q in range(max(key) + 1)]
        passes = [q for q in passes if q]
        pk = max(peak_of(nbytes[q], lo_a[q], hi_a[q], n_frames) for q in passes)
        tried.append((passes, pk))
        if pk <= limit:
            return passes, pk
    low = min(t[1] for t in tried)
    cut = low + 0.05 * (tried[0][1] - low)
    return next(t for t in tried if t[1] <= cut)
