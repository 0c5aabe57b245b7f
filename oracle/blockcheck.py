"""Parity of an integrated phi block on a stratified sample of its rows: TEST INFRASTRUCTURE (see
oracle/__init__.py). Used by the GPU tests and by bench.py after its timed region, as the checker only.

Every sampled row is integrated again by the restatement from the same raw frames: its box window is read from the
frame stack (`crop`), prepared and gathered as XPG's frame loop does (`xpg/integrate.py:648-787`), then pass 1 with
the widths the block's pass 1 used and pass 2 with the block's learnt profiles and adapted widths
(`xpg/integrate.py:521-573`), which the device run reports in `IntegrationResult.block_widths` and `.profiles`.
The rows are drawn from every shoebox shape group (depth, side, phi binning, super-pixel side, partner), so the
sample covers the block's whole mix of launch shapes.
"""
from __future__ import annotations

import numpy as np

from . import gather as OG
from . import kernels as OK

P1_KEYS = ("bg", "isum", "vsum", "vsum0", "xo", "yo", "zo", "frac_rec", "m_d", "m_m")
P2_KEYS = ("iprf", "vprf", "vprf0", "corr", "p_valid", "p_total", "rho", "p_fg")
INT_KEYS = ("n_over", "n_fg_masked", "isum_raw")


def stratified_rows(plan, rows, n_min=500, seed=0):
    """At least n_min of `rows` (or all of them), the same number from every (Dz, bx, fb, pxs, partner) group where
    the group holds that many, topped up at random; sorted."""
    rows = np.asarray(rows, np.int64)
    if rows.size <= n_min:
        return rows
    rng = np.random.default_rng(seed)
    key = np.stack([plan.Dz[rows], plan.bx[rows], plan.fb[rows], plan.pxs[rows],
                    np.asarray(plan.has_partner[rows], np.int64)], 1)
    _, gid = np.unique(key, axis=0, return_inverse=True)
    gid = gid.reshape(-1)
    n_groups = int(gid.max()) + 1
    per = max(int(np.ceil(n_min / n_groups)), 2)
    take = []
    for g in range(n_groups):
        members = np.flatnonzero(gid == g)
        take.append(rng.choice(members, min(per, members.size), replace=False))
    picked = np.unique(np.concatenate(take))
    if picked.size < n_min:
        rest = np.setdiff1d(np.arange(rows.size), picked)
        picked = np.union1d(picked, rng.choice(rest, n_min - picked.size, replace=False))
    return rows[picked]


def _box_frames(crop, plan, j, n_frames, ny, nx, overload):
    """{fi: prepared frame window at the row's super-pixel scale} of every read frame the box reaches, and the
    window's origin in those units."""
    s = int(plan.pxs[j])
    span = int(plan.Dz[j]) * int(plan.fb[j])
    f_lo, f_hi = max(int(plan.iz0[j]), 0), min(int(plan.iz0[j]) + span, n_frames)
    y_lo, x_lo = max(int(plan.iy0[j]) * s, 0), max(int(plan.ix0[j]) * s, 0)
    y_hi = min((int(plan.iy0[j]) + int(plan.bx[j])) * s, ny)
    x_hi = min((int(plan.ix0[j]) + int(plan.bx[j])) * s, nx)
    out = {}
    if f_hi > f_lo and y_hi > y_lo and x_hi > x_lo:
        raw = crop(f_lo, f_hi, y_lo, y_hi, x_lo, x_hi)
        for k in range(f_hi - f_lo):
            pf = OG.prepare_frame(raw[k], overload)
            out[f_lo + k] = pf if s == 1 else OG.superpixel_frame(pf, s)
    return out, (y_lo // s, x_lo // s)


def check_rows(crop, plan, rows, res, block, geom, n_frames, ny, nx, overload, gain, bkg_template=None):
    """Worst error per result key of the device run's rows against the restatement: floats relative to
    max(|value|, scale) as tests/tolerance.py defines it, integers as the count of rows that differ. Returns
    (worst, n_bad, details) with n_bad the rows outside tolerance per key."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "tests"))
    import tolerance as T
    from .pipeline import row_payload
    det = OK.detector_consts(geom, bkg_template)
    s0 = geom.s0.astype(np.float32)
    axis = geom.axis.astype(np.float32)
    phi0 = np.float32(np.radians(geom.z_to_phi(0.0)))
    osc = np.float32(np.radians(geom.osc))
    w = res.block_widths[block]
    (sd1, sm1, rcw1), (sd2, sm2, rcw2) = w["pass1"], w["pass2"]
    prof = np.asarray(res.profiles[block], np.float32)
    refl = res.refl
    worst = {k: 0.0 for k in P1_KEYS + P2_KEYS}
    bad = {k: 0 for k in P1_KEYS + P2_KEYS + INT_KEYS}
    n_fitted = 0
    for (r, nb), j in zip(row_payload(plan, rows), rows):
        frames, (oy, ox) = _box_frames(crop, plan, j, n_frames, ny, nx, overload)
        sb = OG.gather_shoebox(frames, sorted(frames), r["iz0"], r["fbi"], r["Dz"], r["bx"], r["iy0"] - oy,
                               r["ix0"] - ox)
        o1 = OK.pass1(sb, r, nb, det, s0, axis, phi0, osc, sd1, sm1, gain, rcw1)
        pix = dict(zeta=o1["zeta"], J=o1["J"], u1=o1["u1"], u2=o1["u2"], seff=o1["seff"])
        o2 = OK.pass2(sb, r, nb, det, s0, axis, phi0, osc, sd2, sm2, gain, prof, o1["bg"], o1["nbg"], rcw2, pix)
        want = dict(o1, **o2)
        ctx = {k: want[k] for k in ("isum", "vsum", "vprf", "p_valid", "p_total", "m_m", "seff")}
        for k in INT_KEYS:
            bad[k] += int(int(refl[k][j]) != int(want[k]))
        for k in P1_KEYS + P2_KEYS:
            ok, e = T.within(k, refl[k][j], want[k], ctx)
            if T.meaningful(k, ctx):
                worst[k] = max(worst[k], e)
            bad[k] += int(not ok)
        n_fitted += int(T.meaningful("iprf", ctx))
    return worst, bad, dict(rows=int(len(rows)), rows_fitted=n_fitted)
