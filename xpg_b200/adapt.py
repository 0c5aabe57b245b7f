"""Per-block adaptation of the spot widths and the rocking-curve shape, and the spot-width estimate of a sweep,
on the pass-1 outputs of strong reflections: the two float64 sweeps over the strong rows' frames (the sigma_M grid
search, the Gram system of the rocking-curve fit) run on the device, the small solves and medians on the host.

References: `_adapt_block` (`xpg/integrate.py:404-461`), `_fit_rocking_width` (`:1130-1154`), `_nnls_gram`
(`:1095-1104`), `_rocking_resolved` (`:1107-1127`), `_estimate_sigmas` (`:1002-1092`), `rc_basis_np`
(`xpg/integrate_kernels.py:144-151`). The arithmetic is the reference's, in float64, so that the widths handed to
pass 2 and to the next block are the same numbers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
from scipy.special import erf

FG_R = 3.0
RC_C = np.linspace(-3.5, 3.5, 21)
RC_W = 0.25
MAX_DZ = 65
PRIOR_N = 300.0          # shrinkage of the block widths towards the run's widths (strong-reflection equivalents)
PRIOR_RC = 200.0         # prior weight of the Gaussian rocking-curve shape


def rc_default_weights():
    w = np.exp(-0.5 * RC_C ** 2 / (1 - RC_W ** 2))
    return (w / w.sum()).astype(np.float32)


def rc_basis(phi_lo, phi_hi, phi_c, zeta, sm):
    """Frame integrals of every mixture component, (n, Dz, K) float64."""
    s = (sm / np.maximum(np.abs(zeta), 1e-3))[:, None, None]
    sw = s * RC_W * np.sqrt(2.0)
    a = (phi_hi[..., None] - phi_c[:, None, None] - RC_C * s) / sw
    b = (phi_lo[..., None] - phi_c[:, None, None] - RC_C * s) / sw
    return 0.5 * (erf(a) - erf(b))


def _rocking_struct(F, IZ, PH, ZK, g):
    """XiRocking of strong rows: F (n, 65) float64 on the device; iz0 / phi (deg) / zeta host arrays."""
    import torch
    from . import native as N
    from .device import h2d
    dev = F.device
    keep = dict(F=F.contiguous(), iz0=h2d(np.asarray(IZ, np.int32), None, dev), phi=h2d(np.asarray(PH, np.float64),
                None, dev), zeta=h2d(np.asarray(ZK, np.float64), None, dev))
    q = N.XiRocking()
    q.n = int(F.shape[0])
    q.fz, q.iz0, q.phi, q.zeta = (N.ptr(keep[k]) for k in ("F", "iz0", "phi", "zeta"))
    q.phi0, q.osc, q.z_shift = float(g.phi0), float(g.osc), float(g.starting_frame - 1)
    return q, keep


def fit_rocking_width(sel_fit, g, sm_guess, lo_fac=0.2, hi_fac=3.0):
    """Grid search (61 points in log sigma_M) of the frame-integrated Gaussian rocking curve against the per-frame
    intensity fractions of strong reflections; each candidate's cost is one device reduction (xi_rocking_costs).
    sel_fit: list of (fz (n, 65), iz0, phi (deg), zeta) with fz a host array or a device tensor."""
    import torch
    from . import native as N
    from .device import TIMER, h2d
    Fs = [torch.as_tensor(s[0], dtype=torch.float64) for s in sel_fit]
    dev = next((f.device for f in Fs if f.is_cuda), torch.device("cuda"))
    F = (torch.cat([f if f.is_cuda else h2d(f.numpy(), None, dev) for f in Fs]) if Fs
         else torch.zeros((0, MAX_DZ), dtype=torch.float64, device=dev))
    iz0 = np.concatenate([s[1] for s in sel_fit]) if sel_fit else np.zeros(0, np.int32)
    phi = np.concatenate([s[2] for s in sel_fit]) if sel_fit else np.zeros(0)
    zeta = np.concatenate([s[3] for s in sel_fit]) if sel_fit else np.zeros(0)
    grid = sm_guess * np.exp(np.linspace(np.log(lo_fac), np.log(hi_fac), 61))
    q, keep = _rocking_struct(F, iz0, phi, zeta, g)
    grid_t = h2d(np.asarray(grid, np.float64), None, dev)
    cost_t = torch.empty(len(grid), dtype=torch.float64, device=dev)
    lib = N.load()
    with TIMER.span("adapt"):
        N.check(lib.xi_rocking_costs(C.byref(q), N.ptr(grid_t), len(grid), N.ptr(cost_t), N.stream_handle()),
                "xi_rocking_costs")
    costs = cost_t.cpu().numpy()
    best = (np.inf, sm_guess)
    for c, sm in zip(costs, grid):
        if c < best[0]:
            best = (c, sm)
    return float(best[1])


def _rocking_weights(q, sm_new, F, IZ, PH, ZK, g):
    """Non-negative rocking-curve mixture weights at width sm_new (rad): the Gram system of A w = y on the device
    (xi_rocking_gram), solved on its 21 x 21 Cholesky factor; the full least-squares form when the Gram matrix is not
    positive definite."""
    import torch
    from scipy.linalg import LinAlgError, cholesky, solve_triangular
    from scipy.optimize import nnls
    from . import native as N
    from .device import TIMER
    lib = N.load()
    dev = F.device
    ws = torch.empty(max(int(lib.xi_rocking_gram_workspace(C.byref(q))), 1), dtype=torch.uint8, device=dev)
    gram = torch.empty((len(RC_C), len(RC_C)), dtype=torch.float64, device=dev)
    rhs = torch.empty(len(RC_C), dtype=torch.float64, device=dev)
    with TIMER.span("adapt", 3):
        N.check(lib.xi_rocking_gram(C.byref(q), float(sm_new), N.ptr(ws), ws.numel(), N.ptr(gram), N.ptr(rhs),
                                    N.stream_handle()), "xi_rocking_gram")
    G, h = gram.cpu().numpy(), rhs.cpu().numpy()
    try:
        R = cholesky(G)
        return nnls(R, solve_triangular(R.T, h, lower=True))[0]
    except (LinAlgError, ValueError):
        Fh = F.cpu().numpy()
        k = np.asarray(IZ)[:, None] + np.arange(Fh.shape[1])[None]
        lo = g.z_to_phi(k.astype(float))
        hi = g.z_to_phi(k + 1.0)
        lo, hi = np.radians(np.minimum(lo, hi)), np.radians(np.maximum(lo, hi))
        Bm = rc_basis(lo, hi, np.radians(PH), ZK, sm_new)
        tot = np.maximum(Fh.sum(1, keepdims=True), 1e-9)
        A = (Bm * np.sqrt(tot)[:, :, None]).reshape(-1, len(RC_C))
        y = (Fh / tot * np.sqrt(tot)).reshape(-1)
        return nnls(A, y)[0]


def _truncation_factor():
    """<r^2/2> / sigma^2 of a 2D Gaussian inside radius FG_R."""
    return 1.0 - (FG_R ** 2 / 2) * np.exp(-FG_R ** 2 / 2) / (1 - np.exp(-FG_R ** 2 / 2))


def adapt_block(g, strong, sd_run, sm_run, sd_b, sm_b, rcw_b):
    """sigma_M and the rocking-curve weights of this block's pass 2, sigma_D of the next block.

    strong: None, or the block's strong rows in the reference's chunk order: dict F (n, 65) float64 per-frame net
    on the device, phi (deg), zeta_k, iz0, m_d, x, y (host arrays). Returns (sm_new, rcw_new, sd_next or None,
    params dict)."""
    n = 0 if strong is None else int(strong["F"].shape[0])
    if n < 100:
        params = dict(sigma_d=float(np.degrees(sd_b)), sigma_m=float(np.degrees(sm_b)), n=n,
                      rcw=np.asarray(rcw_b).round(3).tolist())
        return sm_b, rcw_b, None, params
    F, PH, ZK, IZ, MD, X, Y = (strong[k] for k in ("F", "phi", "zeta_k", "iz0", "m_d", "x", "y"))
    sm_fit = np.radians(fit_rocking_width([(F, IZ, PH, ZK)], g, np.degrees(sm_run), 0.5, 2.0))
    sm_new = float(np.exp((n * np.log(sm_fit) + PRIOR_N * np.log(sm_run)) / (n + PRIOR_N)))
    q, keep = _rocking_struct(F, IZ, PH, ZK, g)
    w = _rocking_weights(q, sm_new, F, IZ, PH, ZK, g)
    lam = PRIOR_RC / n
    w = (w / max(w.sum(), 1e-9) + lam * rc_default_weights()) / (1 + lam)
    Xv = g.pixel_to_lab(X, Y)
    Xlen = np.linalg.norm(Xv, axis=1)
    cosa = np.abs(Xv @ g.ed3) / Xlen
    md = MD / _truncation_factor() - (g.qx / Xlen) ** 2 * (1 + cosa ** 2) / 24.0
    sd_fit = float(np.clip(np.sqrt(max(np.median(md), 1e-12)), 0.5 * sd_run, 2.0 * sd_run))
    sd_new = float(np.exp((n * np.log(sd_fit) + PRIOR_N * np.log(sd_run)) / (n + PRIOR_N)))
    params = dict(sigma_d=float(np.degrees(sd_b)), sigma_m=float(np.degrees(sm_new)), n=int(n),
                  rcw=w.round(3).tolist(), sigma_d_fit=float(np.degrees(sd_fit)),
                  sigma_m_fit=float(np.degrees(sm_fit)))
    return float(sm_new), w.astype(np.float32), sd_new, params


def rocking_resolved(r, max_edge=0.5):
    """Rows whose per-frame net counts show a rocking curve inside the box (`xpg/integrate.py:1107-1127`): the mean of
    the outermost recorded bins (bins beyond the sweep hold exactly 0) is below `max_edge` times the bin holding the
    predicted centre, with at least three bins between them; boxes under 3 bins always pass."""
    fz = r.get("fz")
    n_rows = len(r["x"])
    if fz is None:
        return np.ones(n_rows, bool)
    depth = fz.shape[1]
    dz = np.minimum(np.asarray(r["dz"], np.int64), depth)
    bins = np.arange(depth)
    recorded = (fz != 0) & (bins[None, :] < dz[:, None])
    lo = np.where(recorded, bins[None, :], depth).min(axis=1)
    hi = np.where(recorded, bins[None, :], -1).max(axis=1)
    none = hi < 0
    lo[none] = 0
    hi[none] = 0
    centre_bin = np.floor((r["z"] - r["iz0"]) / np.maximum(r["fb"], 1)).astype(np.int64)
    centre_bin = np.minimum(np.maximum(centre_bin, 0), np.maximum(dz - 1, 0))
    take = lambda k: np.take_along_axis(fz, k[:, None], axis=1)[:, 0]
    peak = take(centre_bin)
    rim = 0.5 * (take(lo) + take(hi))
    return (dz < 3) | ((peak > 0) & (rim < max_edge * peak) & (hi - lo >= 2))


def _sample_ranges(f0, f1, osc, n_sample_frames, n_ranges=5):
    """The frame ranges the spot widths are measured on: n_ranges evenly spaced ranges of at least 5 degrees (and of
    n_sample_frames / 3 frames), no longer than the sweep's n_ranges-th part."""
    nf = f1 - f0 + 1
    span = max(int(round(n_sample_frames / 3)), int(np.ceil(5.0 / max(abs(osc), 1e-6))), 3)
    span = min(span, max(nf // n_ranges, 3))
    starts = [f0 + int(k * (nf - span) / max(n_ranges - 1, 1)) for k in range(n_ranges)]
    return [(a, min(a + span - 1, f1)) for a in starts]


class _RangeRows:
    """Moment-only results of one sampled range: the rows usable for the width estimate (`base`), their I/sigma,
    and the per-row corrections of the second moments (pixel footprint, frame-bin width)."""

    def __init__(self, r, a, b, g):
        self.r = r
        ok = (r["z"] >= a - 1) & (r["z"] < b) & (r.get("lattice", 0) == 0) & ~r["overlap"]
        ok &= np.isfinite(r["isum"]) & (r["isum"] > 0) & (r["n_over"] == 0) & (r["frac_rec"] > 0.98)
        self.base = ok & rocking_resolved(r)
        self.isig = r["isum"] / np.sqrt(np.maximum(r["vsum"], 1e-6))
        self.g = g

    def count_above(self, t):
        return int((self.base & (self.isig > t)).sum())

    def pick(self, t):
        return self.base & (self.isig > t)

    def moments(self, sel):
        """(m_d, footprint) pairs, frame-width-corrected m_m, and the per-frame fit rows of the selected rows."""
        r, g = self.r, self.g
        lab = g.pixel_to_lab(r["x"][sel], r["y"][sel])
        dist = np.linalg.norm(lab, axis=1)
        cos_in = np.abs(lab @ g.ed3) / dist
        foot = (g.qx / dist) ** 2 * (1 + cos_in ** 2) / 24.0      # pixel footprint per axis (eps units)
        if "pxs" in r:
            foot = foot * r["pxs"][sel] ** 2
        fb = r["fb"][sel] if "fb" in r else 1
        mm = r["m_m"][sel] - (np.radians(g.osc) * fb * r["zeta_k"][sel]) ** 2 / 12.0
        per_frame = sel & (r["fb"] == 1) if "fb" in r else sel
        fit = (r["fz"][per_frame], r["iz0"][per_frame], r["phi"][per_frame], r["zeta_k"][per_frame])
        return np.c_[r["m_d"][sel], foot], mm, fit


def _thresholds(ranges):
    """Per-range I/sigma threshold of the strong rows, or None for a range left out: 20, or 10 where fewer than
    150 rows pass 20; a range with fewer than 20 rows at its threshold is left out. When every range is left out
    and the ranges together hold at least 30 rows above 5, every range takes 5."""
    counts = np.array([[rr.count_above(t) for t in (20.0, 10.0, 5.0)] for rr in ranges]).reshape(-1, 3)
    thr = np.where(counts[:, 0] >= 150, 20.0, 10.0)
    kept = np.where(counts[:, 0] >= 150, counts[:, 0], counts[:, 1]) >= 20
    if not kept.any() and counts[:, 2].sum() >= 30:
        return [5.0] * len(ranges)
    return [float(t) if k else None for t, k in zip(thr, kept)]


def _growing(new, cur, prev):
    """The width estimate grows with the box (both the last step and this one by more than 15%): contamination."""
    up = lambda a, b: a.sigma_d > 1.15 * b.sigma_d or a.sigma_m > 1.15 * b.sigma_m
    return up(new, cur) and up(cur, prev)


def estimate_sigmas(integrate_fn, images, exp, model0, dmin, frames, n_sample_frames=30, verbose=True, log=print,
                    extra_exps=(), bkg_template=None, foreign_spots=None, max_iter=None, guard=None):
    """sigma_D / sigma_M of a sweep from the truncation-corrected second moments and rocking curves of strong spots
    over sampled frame ranges (`xpg/integrate.py:1002-1092`), up to 3 rounds, each round integrating the ranges with
    the previous round's widths. `integrate_fn` is the moments-only integration."""
    from .plan import IntegrationModel
    g = exp.geom
    f0, f1 = frames
    ranges = _sample_ranges(f0, f1, g.osc, n_sample_frames)
    lattices = [[e] for e in extra_exps] or None
    cur = prev = model0
    history = []
    for rnd in range(max_iter or 3):
        stats = []
        for a, b in ranges:
            res = integrate_fn(images, [exp], np.array([a - 1.0, float(b)]), cur, dmin,
                               frames=(max(f0, a - 5), min(f1, b + 5)), verbose=False, learn_profiles=False,
                               adaptive=False, bkg_template=bkg_template, extra_lattices=lattices,
                               foreign_spots=foreign_spots, moments_only=True)
            stats.append(_RangeRows(res.refl, a, b, g))
        picked = [rr.moments(rr.pick(t)) for rr, t in zip(stats, _thresholds(stats))
                  if t is not None and rr.pick(t).any()]
        if not picked:
            break
        md_pairs = np.concatenate([p[0] for p in picked])
        mm = np.concatenate([p[1] for p in picked])
        md = md_pairs[:, 0] / _truncation_factor() - md_pairs[:, 1]
        sd_deg = np.degrees(np.sqrt(max(np.median(md), 1e-12)))
        mm_deg = np.degrees(np.sqrt(max(np.median(mm), 1e-12)))
        sm_deg = fit_rocking_width([p[2] for p in picked], g, max(mm_deg, 0.5 * cur.sigma_m))
        new = IntegrationModel(sigma_d=float(np.clip(sd_deg, 0.005, 1.0)), sigma_m=float(np.clip(sm_deg, 0.005, 5.0)),
                               gain=cur.gain)
        history.append((float(new.sigma_d), float(new.sigma_m), int(md.size)))
        if verbose:
            log(f"  INTEGRATE: estimated sigma_D {new.sigma_d:.4f} deg, sigma_M {new.sigma_m:.4f} deg "
                f"from {md.size} strong spots (iteration {rnd + 1})")
        if (guard is None or guard) and rnd >= 1 and _growing(new, cur, prev):
            if verbose:
                log(f"  INTEGRATE: spot-width estimate keeps growing with the box (contamination): keeping "
                    f"iteration {rnd} values")
            break
        prev, cur = cur, new
        settled = abs(cur.sigma_d / prev.sigma_d - 1) < 0.03 and abs(cur.sigma_m / prev.sigma_m - 1) < 0.03
        if max_iter and rnd >= 2 and settled:
            break
    cur.history = history
    return cur
