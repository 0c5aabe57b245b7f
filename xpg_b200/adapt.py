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
    """Rows whose net counts show a rocking curve inside the box (first and last recorded bins well below the bin
    of the predicted centre)."""
    fz = r.get("fz")
    if fz is None:
        return np.ones(len(r["x"]), bool)
    n = len(fz)
    dz = np.minimum(np.asarray(r["dz"], int), fz.shape[1])
    rows = np.arange(n)
    c = np.clip(np.floor((r["z"] - r["iz0"]) / np.maximum(r["fb"], 1)).astype(int), 0, np.maximum(dz - 1, 0))
    centre = fz[rows, c]
    k = np.arange(fz.shape[1])[None]
    rec = (fz != 0) & (k < dz[:, None])
    first = np.where(rec.any(1), np.argmax(rec, 1), 0)
    last = np.where(rec.any(1), fz.shape[1] - 1 - np.argmax(rec[:, ::-1], 1), 0)
    edge = 0.5 * (fz[rows, first] + fz[rows, last])
    return (dz < 3) | ((centre > 0) & (edge < max_edge * centre) & (last - first >= 2))


def estimate_sigmas(integrate_fn, images, exp, model0, dmin, frames, n_sample_frames=30, verbose=True, log=print,
                    extra_exps=(), bkg_template=None, foreign_spots=None, max_iter=None, guard=None):
    """sigma_D / sigma_M from second moments and rocking curves of strong spots over 5 sampled frame ranges,
    iterated up to 3 times (`xpg/integrate.py:1002-1092`). `integrate_fn` is the moments-only integration."""
    from .plan import IntegrationModel
    g = exp.geom
    f0, f1 = frames
    nf = f1 - f0 + 1
    nr = 5
    span = max(int(round(n_sample_frames / 3)), int(np.ceil(5.0 / max(abs(g.osc), 1e-6))), 3)
    span = min(span, max(nf // nr, 3))
    ranges = []
    for i in range(nr):
        a = f0 + int(i * (nf - span) / max(nr - 1, 1))
        ranges.append((a, min(a + span - 1, f1)))
    model = prev = model0
    history = []
    for it in range(max_iter or 3):
        sel_md, sel_mm, sel_fit, per_range = [], [], [], []
        for a, b in ranges:
            edges = np.array([a - 1.0, float(b)])
            res = integrate_fn(images, [exp], edges, model, dmin, frames=(max(f0, a - 5), min(f1, b + 5)),
                               verbose=False, learn_profiles=False, adaptive=False, bkg_template=bkg_template,
                               extra_lattices=[[e] for e in extra_exps] or None, foreign_spots=foreign_spots,
                               moments_only=True)
            r = res.refl
            z_ok = (r["z"] >= a - 1) & (r["z"] < b) & (r.get("lattice", 0) == 0) & ~r["overlap"]
            isg = r["isum"] / np.sqrt(np.maximum(r["vsum"], 1e-6))
            base = z_ok & np.isfinite(r["isum"]) & (r["isum"] > 0) & (r["n_over"] == 0) & (r["frac_rec"] > 0.98)
            base &= rocking_resolved(r)
            per_range.append((r, base, isg))
        sels = []
        for r, base, isg in per_range:
            strong = base & (isg > 20)
            if strong.sum() < 150:
                strong = base & (isg > 10)
            sels.append(strong if strong.sum() >= 20 else None)
        if all(x is None for x in sels) and sum(int((bs & (ig > 5.0)).sum()) for _, bs, ig in per_range) >= 30:
            sels = [bs & (ig > 5.0) for _, bs, ig in per_range]
        for (r, base, isg), strong in zip(per_range, sels):
            if strong is None or not strong.any():
                continue
            Xv = g.pixel_to_lab(r["x"][strong], r["y"][strong])
            Xlen = np.linalg.norm(Xv, axis=1)
            cosa = np.abs(Xv @ g.ed3) / Xlen
            pix = (g.qx / Xlen) ** 2 * (1 + cosa ** 2) / 24.0
            if "pxs" in r:
                pix = pix * r["pxs"][strong] ** 2
            sel_md.append(np.c_[r["m_d"][strong], pix])
            fbs = r["fb"][strong] if "fb" in r else 1
            sel_mm.append(r["m_m"][strong] - (np.radians(g.osc) * fbs * r["zeta_k"][strong]) ** 2 / 12.0)
            one = strong & (r["fb"] == 1) if "fb" in r else strong
            sel_fit.append((r["fz"][one], r["iz0"][one], r["phi"][one], r["zeta_k"][one]))
        if not sel_md:
            break
        md2 = np.concatenate(sel_md)
        mm = np.concatenate(sel_mm)
        md = md2[:, 0] / _truncation_factor() - md2[:, 1]
        sd_new = np.degrees(np.sqrt(max(np.median(md), 1e-12)))
        sm_new = fit_rocking_width(sel_fit, g, max(np.degrees(np.sqrt(max(np.median(mm), 1e-12))),
                                                  0.5 * model.sigma_m))
        new = IntegrationModel(sigma_d=float(np.clip(sd_new, 0.005, 1.0)), sigma_m=float(np.clip(sm_new, 0.005, 5.0)),
                               gain=model.gain)
        history.append((float(new.sigma_d), float(new.sigma_m), int(md.size)))
        if verbose:
            log(f"  INTEGRATE: estimated sigma_D {new.sigma_d:.4f} deg, sigma_M {new.sigma_m:.4f} deg "
                f"from {md.size} strong spots (iteration {it + 1})")
        if (guard is None or guard) and it >= 1 and (new.sigma_d > 1.15 * model.sigma_d
                                                      or new.sigma_m > 1.15 * model.sigma_m) and \
                (model.sigma_d > 1.15 * prev.sigma_d or model.sigma_m > 1.15 * prev.sigma_m):
            if verbose:
                log(f"  INTEGRATE: spot-width estimate keeps growing with the box (contamination): keeping "
                    f"iteration {it} values")
            break
        prev, model = model, new
        if max_iter and it >= 2 and abs(model.sigma_d / prev.sigma_d - 1) < 0.03 and \
                abs(model.sigma_m / prev.sigma_m - 1) < 0.03:
            break
    model.history = history
    return model
