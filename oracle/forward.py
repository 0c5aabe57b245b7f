"""CPU restatement of the forward-model likelihood passes (TEST INFRASTRUCTURE: the checker of the library's
xi_fm_scatter / xi_fm_gather, never product code).

XPG's pixel-level forward model (xpg/forward/) keeps, per chunk of reflections, separable profile factors: a
reflection's fraction in voxel (z, y, x) of its box is f = sum_t R[t, row, z] * P[t, row, y, x] (the product of a
rocking-curve factor and a detector-profile factor per term; `expand_terms`, xpg/forward/model.py:197-203). The
voxels of a window of frames [f0, f1) x rows [y0, y0 + ny) x columns [x0, x0 + nx) are indexed densely,
(kz * ny + ky) * nx + kx with kz = iz0 + z - f0, ky = iy0 + y - y0, kx = ix0 + x - x0; voxels outside the window are
dropped (`WindowModel.vid`, :381-392). The passes (`WindowModel.mu`, `grad_ratio`, `grad_newton`, :476-577; fused
on CUDA by the Triton kernels of xpg/forward/kernels.py:34-103):

    scatter:       mu[v] += I_row * f + beta_row                 over every in-window voxel of each box
    grad_ratio:    g[row] += sum f * A[v] / M[v]                 over in-window voxels with NS[v] >= 0
    grad_newton:   g[row] += sum f * (1 - max(NS[v], 0) / M[v]), fd[row] += sum f^2 / max(M[v], 1e-6)   (same voxels)

The separable factors themselves (`fraction_terms`, model.py:206-280) are restated below as well, one reflection at
a time on the pass-1 geometry of oracle.kernels (pinned on XPG's own factors: tests/golden/forward_terms.npz).

f and every product are float32 as XPG computes them (separate roundings, no fused multiply-add); the sums are
accumulated in float64 here (XPG's and the device's float32 sums differ from them by float32 rounding in another
order, which the tests' tolerance covers). Pinned on XPG's own passes run on the same inputs
(tests/golden/forward.npz, made by tests/golden/make_forward_golden.py).
"""
from __future__ import annotations

import numpy as np


def fractions(R, P):
    """f (n, Dz, b, b) float32 = sum_t R[t][:, :, None, None] * P[t][:, None] (products rounded, then summed)."""
    f = None
    for t in range(R.shape[0]):
        g = (R[t][:, :, None, None] * P[t][:, None]).astype(np.float32)
        f = g if f is None else (f + g).astype(np.float32)
    return f


def voxel_index(iz0, iy0, ix0, Dz, b, win):
    """Dense window index (n, Dz, b, b) of every box voxel, -1 outside the window."""
    f0, f1, y0, ny, x0, nx = (int(v) for v in win)
    kz = np.asarray(iz0, np.int64)[:, None] + np.arange(Dz)[None] - f0
    ky = np.asarray(iy0, np.int64)[:, None] + np.arange(b)[None] - y0
    kx = np.asarray(ix0, np.int64)[:, None] + np.arange(b)[None] - x0
    ok = ((kz >= 0) & (kz < f1 - f0))[:, :, None, None] & ((ky >= 0) & (ky < ny))[:, None, :, None] \
        & ((kx >= 0) & (kx < nx))[:, None, None, :]
    lin = (kz[:, :, None, None] * ny + ky[:, None, :, None]) * nx + kx[:, None, None, :]
    return np.where(ok, lin, -1)


def scatter(mu, groups, I, beta, win):
    """mu (float64 copy of the window's starting values) += I f + beta over each group's in-window voxels. groups:
    dicts of R (T, n, Dz), P (T, n, b, b), iz0, iy0, ix0, rows."""
    out = np.asarray(mu, np.float64).copy()
    for g in groups:
        R, P = g["R"], g["P"]
        f = fractions(R, P)
        v = voxel_index(g["iz0"], g["iy0"], g["ix0"], R.shape[2], P.shape[-1], win)
        val = (f * I[g["rows"]][:, None, None, None]).astype(np.float32)
        if beta is not None and len(beta):
            val = (val + beta[g["rows"]][:, None, None, None]).astype(np.float32)
        ok = v >= 0
        np.add.at(out, v[ok], val[ok].astype(np.float64))
    return out


def gather(groups, win, n, A, M, NS, mode):
    """mode 0: g[row] = sum f A / M; mode 1: g[row] = sum f (1 - max(NS, 0) / M), fd[row] = sum f^2 / max(M, 1e-6);
    over each box's in-window voxels with NS >= 0. Returns (g, fd) float64 (fd None for mode 0)."""
    g_out = np.zeros(n, np.float64)
    fd_out = np.zeros(n, np.float64) if mode == 1 else None
    for g in groups:
        R, P = g["R"], g["P"]
        f = fractions(R, P)
        v = voxel_index(g["iz0"], g["iy0"], g["ix0"], R.shape[2], P.shape[-1], win)
        vc = np.maximum(v, 0)
        ns = np.asarray(NS)[vc].astype(np.float32)
        use = (v >= 0) & (ns >= 0)
        m = np.asarray(M, np.float32)[vc]
        if mode == 0:
            w = (np.asarray(A, np.float32)[vc] / m).astype(np.float32)
        else:
            w = (np.float32(1.0) - (np.maximum(ns, np.float32(0.0)) / m).astype(np.float32)).astype(np.float32)
            d = ((f * f).astype(np.float32) / np.maximum(m, np.float32(1e-6))).astype(np.float32)
            np.add.at(fd_out, g["rows"], np.where(use, d, 0.0).astype(np.float64).sum(axis=(1, 2, 3)))
        t = (f * w).astype(np.float32)
        np.add.at(g_out, g["rows"], np.where(use, t, 0.0).astype(np.float64).sum(axis=(1, 2, 3)))
    return g_out, fd_out


# ---- separable factors (`fraction_terms`, xpg/forward/model.py:206-280) ---------------------------------------

def _phi_rc(lo, hi, phi, zeta, sm, rcw=None):
    """Rocking-curve fraction recorded between lo and hi (`_phi_rc`, xpg/integrate_kernels.py:130-141): a Gaussian of
    scale sm / |zeta|, or the mixture of RC_C-shifted components weighted by rcw (float32, components summed in
    float64)."""
    from .kernels import RC_C, RC_W, SQRT2_F32
    from .fp import F32, F64, erf32, f32
    s = F32(sm) / np.maximum(np.abs(F32(zeta)), F32(1e-3))
    if rcw is None:
        a = (hi - F32(phi)) / (s * SQRT2_F32)
        b = (lo - F32(phi)) / (s * SQRT2_F32)
        return f32(F32(0.5) * (erf32(a) - erf32(b)))
    c = RC_C.astype(F32)
    sw = (s * F32(RC_W)) * SQRT2_F32
    a = ((hi[:, None] - F32(phi)) - c * s) / sw
    b = ((lo[:, None] - F32(phi)) - c * s) / sw
    term = (f32(rcw) * F32(0.5)) * (erf32(a) - erf32(b))
    return term.astype(F64).sum(axis=1).astype(F32)


def fraction_terms(det, S, phi, ix0, iy0, iz0, Dz, b, s0, axis, frames_phi0, osc, sd, sm, prof=None, region=None,
                   umax=4.5, halo=None, rcw=None):
    """[(R (n, Dz), P (n, b, b)), ...] of the reflections (one term; two with the halo (w, kappa)), one reflection
    at a time: Kabsch frame and eps1 / eps2 of each box pixel, the pixel's solid angle J from the second-order
    gradients of eps, the rocking-curve fractions of the box's frames, and the detector profile, either the
    parametric Gaussian of width seff (sigma_D widened by the pixel) or the learnt profile of the reflection's
    region sampled bilinearly in units of seff within +-umax."""
    from .fp import F32, f32
    from .kernels import box_coords, eps12, kabsch_frame, pixel_area
    n = len(phi)
    G = prof.shape[-1] if prof is not None else 0
    Rs, Ps, Rh_s, Ph_s = [], [], [], []
    for j in range(n):
        r = dict(ix0=int(ix0[j]), iy0=int(iy0[j]), iz0=int(iz0[j]), fb=1.0)
        x, y, _ = box_coords(r, Dz, b, b)
        e1, e2, zeta = kabsch_frame(f32(S[j]), f32(s0), f32(axis))
        eps1, eps2 = eps12(det, f32(S[j]), e1, e2, x, y)
        J = pixel_area(eps1, eps2)
        k = (F32(iz0[j]) + np.arange(Dz, dtype=F32)).astype(F32)
        lo = (F32(frames_phi0) + F32(osc) * k).astype(F32)
        hi = (lo + F32(osc)).astype(F32)
        lo, hi = np.minimum(lo, hi), np.maximum(lo, hi)
        R = _phi_rc(lo, hi, phi[j], zeta, sm, rcw)
        pix = np.sqrt(J[b // 2, b // 2]).astype(F32)
        seff = F32(F32(sd) * np.sqrt(F32(1.0) + (pix / F32(sd)) ** 2 / F32(12.0)))
        r2 = (eps1 * eps1 + eps2 * eps2).astype(F32)

        def gauss2(se):
            return f32(np.exp(F32(-0.5) * r2 / (se * se)) / F32(2 * np.pi) * J / (se * se))
        if prof is None:
            P = gauss2(seff)
        else:
            u1, u2 = (eps1 / seff).astype(F32), (eps2 / seff).astype(F32)
            g1 = ((u1 + F32(umax)) / F32(2 * umax) * F32(G - 1)).astype(F32)
            g2 = ((u2 + F32(umax)) / F32(2 * umax) * F32(G - 1)).astype(F32)
            inside = (g1 >= 0) & (g1 <= G - 1) & (g2 >= 0) & (g2 <= G - 1)
            g1 = np.clip(g1, F32(0), F32(G - 1 - 1e-4))
            g2 = np.clip(g2, F32(0), F32(G - 1 - 1e-4))
            i1, i2 = np.floor(g1).astype(np.int64), np.floor(g2).astype(np.int64)
            t1, t2 = (g1 - i1).astype(F32), (g2 - i2).astype(F32)
            pr = f32(prof[int(region[j])])
            v = ((F32(1) - t1) * (F32(1) - t2) * pr[i2, i1] + t1 * (F32(1) - t2) * pr[i2, i1 + 1]
                 + (F32(1) - t1) * t2 * pr[i2 + 1, i1] + t1 * t2 * pr[i2 + 1, i1 + 1])
            P = f32(np.where(inside, v, F32(0)) * J / (seff * seff))
        if halo is not None:
            w, kap = (F32(v_) for v_ in halo)
            sh = F32(np.sqrt((kap * F32(sd)) ** 2 + pix * pix / F32(12.0)))
            Rh_s.append(f32(w * _phi_rc(lo, hi, phi[j], zeta, F32(kap) * F32(sm))))
            Ph_s.append(gauss2(sh))
            R = f32((F32(1) - w) * R)
        Rs.append(R)
        Ps.append(P)
    terms = [(np.stack(Rs), np.stack(Ps))]
    if halo is not None:
        terms.append((np.stack(Rh_s), np.stack(Ph_s)))
    return terms
