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


def row_bytes(plan):
    """Device bytes of every row while its block is open: the shoebox (value + 3 floats, rows on 16 bytes, and the
    buffer pool's 5% slack), bin counters of binned rows, the per-pixel pass-1 tables (img2, J, u1, u2,
    all_valid2), per-frame fz, per-row scalars of both passes."""
    Dz = plan.Dz.astype(np.int64)
    bx = plan.bx.astype(np.int64)
    arena = 4 * ((Dz * bx * bx + 3) & ~3)
    return (arena + arena // 20 + np.where(plan.fb > 1, 4 * Dz, 0) + 17 * bx * bx + 4 * Dz + 400)   # + the pool's 5%


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


def split_blocks(blocks_refl, z, w_row, k):
    """Every block's rows in k parts of consecutive z with about equal bytes (rows in index order within a part;
    empty parts dropped): (parts, the block of each part)."""
    parts, parent = [], []
    for b, rows in enumerate(blocks_refl):
        if not rows.size:
            continue
        o = rows[np.argsort(z[rows], kind="stable")]
        c = np.cumsum(w_row[o])
        cuts = np.searchsorted(c, c[-1] * np.arange(1, k) / k, side="right")
        for part in np.split(o, cuts):
            if part.size:
                parts.append(np.sort(part))
                parent.append(b)
    return parts, parent


def fit(plan, exp_blocks, n_frames, wedge_bytes, limit, allow_passes=True):
    """The plan (and per-block experiments) whose open blocks fit `limit` bytes with the wedge buffers: unchanged
    when it fits, else every block split into the fewest parts (2..8) that fit, or the split with the lowest peak;
    when that still does not fit (boxes deeper than a block: parts of a block stay open together) and the frames can
    be read again (allow_passes), the blocks go in several passes over the frames (info["passes"]).
    Returns (plan, exp_blocks, info)."""
    w_row = row_bytes(plan)
    one, big = peak_bytes(plan.blocks_refl, plan.need_lo, plan.need_hi, w_row, n_frames)
    info = dict(peak=one + wedge_bytes, one=one + wedge_bytes, parts=1, budget=limit)
    if limit is None or one + wedge_bytes <= limit:
        return plan, exp_blocks, info
    best = None
    for k in range(2, BLOCK_PARTS_MAX + 1):
        parts, parent = split_blocks(plan.blocks_refl, plan.refl["z"], w_row, k)
        lo = [int(plan.zstart[r].min()) for r in parts]
        hi = [int(plan.zend[r].max()) for r in parts]
        pk, _ = peak_bytes(parts, lo, hi, w_row, n_frames)
        if best is None or pk < best[0]:
            best = (pk, k, parts, parent, lo, hi)
        if pk + wedge_bytes <= limit:
            break
    pk, k, parts, parent, lo, hi = best
    if pk < one:
        plan = replace(plan, blocks_refl=parts, need_lo=lo, need_hi=hi)
        exp_blocks = [exp_blocks[b] for b in parent]
        info.update(peak=pk + wedge_bytes, parts=k, parent=parent)
    if info["peak"] > limit and allow_passes:
        passes, ppk = split_passes(plan, w_row, n_frames, limit - wedge_bytes)
        if len(passes) > 1:
            info.update(peak=ppk + wedge_bytes, passes=passes)
    return plan, exp_blocks, info


def split_passes(plan, w_row, n_frames, limit, max_passes=16):
    """Passes over the frames, each integrating the blocks m apart in phi (XPG's grouping along phi,
    `_plan_passes`, xpg/shoebox.py:134-196): the fewest passes whose open blocks fit `limit`, else the lowest peak.
    Returns (passes: block lists, their peak)."""
    blocks = [b for b in range(len(plan.blocks_refl)) if plan.blocks_refl[b].size]
    best = None
    for m in range(2, max_passes + 1):
        passes = [[b for k, b in enumerate(blocks) if k % m == r] for r in range(m)]
        passes = [q for q in passes if q]
        pk = max(peak_bytes([plan.blocks_refl[b] for b in q], [plan.need_lo[b] for b in q],
                            [plan.need_hi[b] for b in q], w_row, n_frames)[0] for q in passes)
        if best is None or pk < best[1]:
            best = (passes, pk)
        if pk <= limit:
            break
    return best
