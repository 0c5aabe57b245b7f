"""Oracle of the per-reflection integration kernels: pixel geometry, pass 1, profile accumulation and finalisation,
pass 2. One reflection at a time; arrays are (Dz, Dy, Dx) float32. TEST INFRASTRUCTURE (see oracle/__init__.py).

Reference: `xpg/integrate_kernels.py` (function by function, cited below).
"""
from __future__ import annotations

import numpy as np

from .fp import (F32, F64, cross3, dot3_fma, dot3_seq, erf32, exp32, expm1_32, f32, norm3, sum32, sum64)

N_FG = 3.0
N_BOX = 5.0
FG_R2 = 9.0                  # FG_R ** 2
BG_R2 = 12.25                # (N_FG + 0.5) ** 2
PROFILE_GRID = 41
UMAX = 4.5                   # N_BOX * 0.9
N_IRLS = 6
VAR_FLOOR = 1e-3
RC_C = np.linspace(-3.5, 3.5, 21)
RC_W = 0.25
SQRT2_F32 = F32(np.sqrt(2.0))


def rc_default_weights():
    """Mixture weights of the unit Gaussian rocking curve (`xpg/integrate_kernels.py:125-127`)."""
    w = np.exp(-0.5 * RC_C ** 2 / (1 - RC_W ** 2))
    return (w / w.sum()).astype(np.float32)


def gaussian_profile(G=PROFILE_GRID):
    """Unit 2D Gaussian on the profile grid (`xpg/integrate_kernels.py:491-495`)."""
    u = np.linspace(-UMAX, UMAX, G)
    U1, U2 = np.meshgrid(u, u)
    return (np.exp(-0.5 * (U1 ** 2 + U2 ** 2)) / (2 * np.pi)).astype(np.float32)


# ------------------------------------------------------------------------------------------------------------------
# detector constants (`xpg/integrate_kernels.py:48-65`)
# ------------------------------------------------------------------------------------------------------------------

def detector_consts(g, bkg_template=None):
    P0, Bx, By = g.panels()
    U1, U2 = Bx / g.qx, By / g.qy
    segmap = g.segmap() if getattr(g, "segmented", False) else None
    geo = getattr(g, "geo_corr", None)
    return dict(orgx=float(g.orgx), orgy=float(g.orgy), qx=float(g.qx), qy=float(g.qy),
                P0=f32(P0), Bx=f32(Bx), By=f32(By), U1=f32(U1), U2=f32(U2), UN=f32(np.cross(U1, U2)),
                segmap=segmap, gx=None if geo is None else f32(geo[0]), gy=None if geo is None else f32(geo[1]),
                wl=float(g.wavelength), tsens=float(max(g.sensor_thickness, 1e-6)), mu=float(max(g.mu, 1e-6)),
                plx=bool(g.has_parallax), bkg=None if bkg_template is None else f32(bkg_template))


def _table_bilinear(tab, x, y):
    """`xpg/detector.py:133-144` in float32."""
    ny, nx = tab.shape
    fx = np.clip(x - F32(1.0), F32(0), F32(nx - 1.000001))
    fy = np.clip(y - F32(1.0), F32(0), F32(ny - 1.000001))
    ix = np.floor(fx).astype(np.int32)
    iy = np.floor(fy).astype(np.int32)
    ix1 = np.minimum(ix + 1, nx - 1)
    iy1 = np.minimum(iy + 1, ny - 1)
    tx = (fx - ix.astype(F32)).astype(F32)
    ty = (fy - iy.astype(F32)).astype(F32)
    one = F32(1.0)
    a = tab[iy, ix] * (one - tx) * (one - ty)
    b = tab[iy, ix1] * tx * (one - ty)
    c = tab[iy1, ix] * (one - tx) * ty
    d = tab[iy1, ix1] * tx * ty
    return ((a + b) + c) + d


def pixel_S(det, x, y):
    """Diffracted wave vector of detector points (`xpg/integrate_kernels.py:78-105`); x, y float32 of equal shape."""
    x = f32(x)
    y = f32(y)
    if det["segmap"] is None:
        P0, Bx, By, U1, U2, UN = (det[n][0] for n in ("P0", "Bx", "By", "U1", "U2", "UN"))
    else:
        sm = det["segmap"]
        ix = np.clip(np.floor(x - F32(0.5)).astype(np.int32), 0, sm.shape[1] - 1)
        iy = np.clip(np.floor(y - F32(0.5)).astype(np.int32), 0, sm.shape[0] - 1)
        k = np.maximum(sm[iy, ix], 0).astype(np.int64)
        P0, Bx, By = det["P0"][k], det["Bx"][k], det["By"][k]
        U1, U2, UN = det["U1"][k], det["U2"][k], det["UN"][k]
    if det["gx"] is None:
        xc, yc = x, y
    else:
        xc = x + _table_bilinear(det["gx"], x, y)
        yc = y + _table_bilinear(det["gy"], x, y)
    orgx, orgy = F32(det["orgx"]), F32(det["orgy"])

    def plane(xx, yy):
        a = (xx - orgx)[..., None]
        b = (yy - orgy)[..., None]
        return ((P0 + a * Bx) + b * By).astype(F32)

    X = plane(xc, yc)
    if det["plx"]:
        tsens, mu = F32(det["tsens"]), F32(det["mu"])
        inv_mu = F32(1.0 / det["mu"])
        qx, qy = F32(det["qx"]), F32(det["qy"])
        for _ in range(2):
            e = X / norm3(X)[..., None]
            cosa = np.clip(dot3_seq_v(e, UN), F32(1e-3), F32(1.0))
            L = tsens / cosa
            muL = mu * L
            lbar = inv_mu - (L * exp32(-muL)) / np.maximum(-expm1_32(-muL), F32(1e-12))
            d1 = lbar * dot3_seq_v(e, U1)
            d2 = lbar * dot3_seq_v(e, U2)
            X = plane(xc - d1 / qx, yc - d2 / qy)
    return (X / (norm3(X) * F32(det["wl"]))[..., None]).astype(F32)


def dot3_seq_v(e, v):
    """Sequential dot product of (..., 3) with (..., 3) or (3,): torch's sum over a length-3 last dimension."""
    p = (e * v).astype(F32)
    return ((p[..., 0] + p[..., 1]) + p[..., 2]).astype(F32)


def bkg_ref(det, x, y):
    """Background template at the pixel centres (`xpg/integrate_kernels.py:68-75`): (Dy, Dx)."""
    if det["bkg"] is None:
        return np.ones((y.size, x.size), F32)
    ny, nx = det["bkg"].shape
    ix = np.clip(np.rint(x - F32(1.0)).astype(np.int32), 0, nx - 1)
    iy = np.clip(np.rint(y - F32(1.0)).astype(np.int32), 0, ny - 1)
    return det["bkg"][iy[:, None], ix[None, :]]


# ------------------------------------------------------------------------------------------------------------------
# per-reflection geometry (`xpg/integrate_kernels.py:219-276`)
# ------------------------------------------------------------------------------------------------------------------

def box_coords(r, Dz, Dy, Dx):
    """Pixel-centre coordinates of the box columns / rows and the frame-bin centres (`:224-230`, `:303`)."""
    if r.get("pxs", 1) > 1:
        s = F32(r["pxs"])
        x = (F32(r["ix0"]) + np.arange(Dx, dtype=F32)) * s + (s - F32(1)) * F32(0.5) + F32(1.0)
        y = (F32(r["iy0"]) + np.arange(Dy, dtype=F32)) * s + (s - F32(1)) * F32(0.5) + F32(1.0)
    else:
        x = F32(r["ix0"]) + np.arange(Dx, dtype=F32) + F32(1.0)
        y = F32(r["iy0"]) + np.arange(Dy, dtype=F32) + F32(1.0)
    fb = F32(r["fb"])
    zz = F32(r["iz0"]) + fb * (np.arange(Dz, dtype=F32) + F32(0.5))
    return f32(x), f32(y), f32(zz)


def kabsch_frame(S, s0, axis):
    """e1, e2 and zeta of a reflection (`:234-238`)."""
    c1 = cross3(S, s0)
    e1 = (c1 / norm3(c1)).astype(F32)
    c2 = cross3(S, e1)
    e2 = (c2 / norm3(c2)).astype(F32)
    zeta = dot3_seq(e1, axis)
    return e1, e2, F32(zeta)


def eps12(det, S, e1, e2, x, y):
    """eps1, eps2 (radians) of the box pixels (`:108-115`): (Dy, Dx)."""
    X, Y = np.meshgrid(x, y)
    Sp = pixel_S(det, X, Y)
    d = (Sp - S).astype(F32)
    invS = F32(1.0) / norm3(S)
    return (dot3_fma(d, e1) * invS).astype(F32), (dot3_fma(d, e2) * invS).astype(F32)


def gradient2(f, axis):
    """Second-order differences with one-sided second-order edges (torch.gradient, edge_order=2, unit spacing)."""
    f = f32(f)
    g = np.empty_like(f)
    sl = lambda i: tuple(slice(None) if a != axis else i for a in range(f.ndim))
    g[sl(slice(1, -1))] = (f[sl(slice(2, None))] - f[sl(slice(None, -2))]) / F32(2.0)
    g[sl(0)] = (F32(-1.5) * f[sl(0)] + F32(2.0) * f[sl(1)]) - F32(0.5) * f[sl(2)]
    g[sl(-1)] = (F32(0.5) * f[sl(-3)] - F32(2.0) * f[sl(-2)]) + F32(1.5) * f[sl(-1)]
    return g


def pixel_area(eps1, eps2):
    """J = |d eps1/dx d eps2/dy - d eps2/dx d eps1/dy| (`:245-248`)."""
    g1x, g1y = gradient2(eps1, 1), gradient2(eps1, 0)
    g2x, g2y = gradient2(eps2, 1), gradient2(eps2, 0)
    return np.abs(g1x * g2y - g2x * g1y).astype(F32)


def rocking_curve(r, Dz, zeta, frames_phi0, osc, sm, rcw):
    """Frame-bin fractions R (Dz,) of the rocking-curve mixture and the bin centres phi_c (`:255-262`, `:130-141`).

    The 21 component terms are summed in float64 in component order and rounded once."""
    fb = F32(r["fb"])
    k = F32(r["iz0"]) + fb * np.arange(Dz, dtype=F32)
    phi_lo = F32(frames_phi0) + F32(osc) * k
    phi_hi = phi_lo + F32(osc) * fb
    lo, hi = np.minimum(phi_lo, phi_hi), np.maximum(phi_lo, phi_hi)
    s = F32(sm) / np.maximum(np.abs(F32(zeta)), F32(1e-3))
    sw = (s * F32(RC_W)) * SQRT2_F32
    c = RC_C.astype(F32)
    phi = F32(r["phi"])
    a = ((hi[:, None] - phi) - c * s) / sw
    b = ((lo[:, None] - phi) - c * s) / sw
    term = (f32(rcw) * F32(0.5)) * (erf32(a) - erf32(b))
    acc = np.zeros(Dz, F64)
    for j in range(term.shape[1]):
        acc = acc + term[:, j].astype(F64)
    R = acc.astype(F32)
    return R, (F32(0.5) * (lo + hi)).astype(F32)


def geometry(det, r, shape, s0, axis, frames_phi0, osc, sd, sm, rcw, pix=None):
    """Per-reflection pixel mapping (`:219-276`). `pix`: pass 1's per-pixel terms (zeta, J, u1, u2, seff)."""
    Dz, Dy, Dx = shape
    x, y, zz = box_coords(r, Dz, Dy, Dx)
    if pix is None:
        if Dx < 3 or Dy < 3:
            raise ValueError("boxes under 3 pixels are not supported")
        e1, e2, zeta = kabsch_frame(f32(r["S"]), f32(s0), f32(axis))
        eps1, eps2 = eps12(det, f32(r["S"]), e1, e2, x, y)
        J = pixel_area(eps1, eps2)
        psz = np.sqrt(J[Dy // 2, Dx // 2])
        sdf = F32(sd)
        q = psz / sdf
        seff = F32(sdf * np.sqrt(F32(1.0) + (q * q) / F32(12.0)))
        u1 = (eps1 / seff).astype(F32)
        u2 = (eps2 / seff).astype(F32)
    else:
        zeta, J, u1, u2, seff = F32(pix["zeta"]), f32(pix["J"]), f32(pix["u1"]), f32(pix["u2"]), F32(pix["seff"])
    R, phi_c = rocking_curve(r, Dz, zeta, frames_phi0, osc, sm, rcw)
    return dict(x=x, y=y, zz=zz, u1=u1, u2=u2, J=J, R=R, zeta=zeta, phi_c=phi_c, seff=seff)


def neighbour_mask(x, y, zz, nb, skip_first=False):
    """Voxels inside any neighbour's foreground ellipsoid (`:186-213`): (Dz, Dy, Dx) bool. The per-voxel test
    ((dx^2 + dy^2) + dz^2 < 1) is separable in its operands, which are computed per column, row and frame."""
    m = np.zeros((zz.size, y.size, x.size), bool)
    for k in range(len(nb["x"])):
        if k == 0 and skip_first:
            continue
        sx, sz = F32(nb["sx"][k]), F32(nb["sz"][k])
        dx = (x - F32(nb["x"][k])) / sx
        dy = (y - F32(nb["y"][k])) / sx
        dz = (zz - F32(nb["z"][k])) / sz
        dxy = (dy * dy)[:, None] + 0 * dx[None, :]
        dxy = ((dx * dx)[None, :] + (dy * dy)[:, None]).astype(F32)
        m |= (dxy[None] + (dz * dz)[:, None, None]) < F32(1.0)
    return m


# ------------------------------------------------------------------------------------------------------------------
# pass 1 (`xpg/integrate_kernels.py:287-365`)
# ------------------------------------------------------------------------------------------------------------------

def pass1(sb, r, nb, det, s0, axis, frames_phi0, osc, sd, sm, gain, rcw):
    """Background, summation, centroids, moments and the projected 2D spot of one reflection."""
    sb = f32(sb)
    Dz, Dy, Dx = sb.shape
    gt = geometry(det, r, sb.shape, s0, axis, frames_phi0, osc, sd, sm, rcw)
    gain = F32(gain)
    valid = sb >= 0
    recorded = sb > F32(-2.5)
    over = sb == F32(-2)
    r2 = (gt["u1"] * gt["u1"] + gt["u2"] * gt["u2"]).astype(F32)
    fg2 = r2 <= F32(FG_R2)
    Rmax = gt["R"].max()
    fgz = gt["R"] >= F32(1e-3) * Rmax + F32(1e-6)
    fg = fg2[None] & fgz[:, None, None]
    nbm = neighbour_mask(gt["x"], gt["y"], gt["zz"], nb)
    bgm = valid & ~fg & ~nbm & (r2 >= F32(BG_R2))[None]
    c = np.where(valid, sb, F32(0)).astype(F32)
    bref = bkg_ref(det, gt["x"], gt["y"])
    w = bgm
    b = sum32(np.where(w, c, 0)) / np.maximum(sum32(np.where(w, bref[None], 0)), F32(1e-6))
    for _ in range(4):
        bp = F32(b) * bref
        thr = (bp + F32(3.0) * np.sqrt(gain * np.maximum(bp, F32(0.5)))) + F32(1.0)
        w = bgm & (c <= thr[None])
        b = sum32(np.where(w, c, 0)) / np.maximum(sum32(np.where(w, bref[None], 0)), F32(1e-6))
    b = F32(b)
    nbg = sum32(np.where(w, bref[None], 0))
    fgv = fg & valid & ~nbm
    bpix = (b * bref).astype(F32)
    net = (c - bpix[None]).astype(F32)
    nfg = F32(fgv.sum())
    sfb = sum32(np.where(fgv, bref[None], 0))
    isum = sum32(np.where(fgv, net, 0))
    isum_raw = int(np.where(fgv, c, F32(0)).astype(np.int64).sum())    # counts are integers: an exact sum
    tail = ((sfb * sfb) * gain) * np.maximum(b, F32(VAR_FLOOR)) / np.maximum(nbg, F32(1.0))
    vsum = gain * sum32(np.where(fgv, c, 0)) + tail
    vsum0 = gain * sum32(np.where(fgv, np.broadcast_to(bpix, c.shape), 0)) + tail
    wpos = np.where(fgv, np.maximum(net, F32(0)), F32(0)).astype(F32)
    sw = np.maximum(sum32(wpos), F32(1e-6))
    xo = sum32(wpos * gt["x"][None, None, :]) / sw
    yo = sum32(wpos * gt["y"][None, :, None]) / sw
    zo = sum32(wpos * gt["zz"][:, None, None]) / sw
    seff = gt["seff"]
    eps1 = (gt["u1"] * seff).astype(F32)
    eps2 = (gt["u2"] * seff).astype(F32)
    wsg = np.where(fgv, net, F32(0)).astype(F32)
    sws = np.maximum(sum32(wsg), F32(1e-6))
    mu1 = sum32(wsg * eps1[None]) / sws
    mu2 = sum32(wsg * eps2[None]) / sws
    e12 = (eps1 * eps1 + eps2 * eps2).astype(F32)
    m_d = ((sum32(wsg * e12[None]) / sws - mu1 * mu1) - mu2 * mu2) / F32(2.0)
    e3 = (gt["zeta"] * (gt["phi_c"] - F32(r["phi"]))).astype(F32)
    mu3 = sum32(wsg * e3[:, None, None]) / sws
    m_m = sum32(wsg * (e3 * e3)[:, None, None]) / sws - mu3 * mu3
    clean = valid & ~nbm
    use_net = np.where(fgz[:, None, None] & clean, net, F32(0))
    okv = clean | ~fgz[:, None, None]
    img2 = sum32(use_net, axis=0)
    all_valid2 = okv.all(axis=0)
    frac_rec = sum32(np.where(recorded.any(axis=(1, 2)), gt["R"], F32(0)))
    n_over = int((over & fg).sum())
    n_fg_masked = int((fg & ~valid & recorded).sum())
    n_fg_nb = int((fg & nbm).sum())
    fz = sum32(np.where(fg2[None] & valid & ~nbm, net, F32(0)), axis=(1, 2))
    return dict(bg=b, nbg=nbg, isum=isum, vsum=F32(vsum), vsum0=F32(vsum0), xo=F32(xo), yo=F32(yo), zo=F32(zo),
                m_d=F32(m_d), m_m=F32(m_m), fz=fz, img2=img2, all_valid2=all_valid2, frac_rec=frac_rec,
                n_over=n_over, n_fg_masked=n_fg_masked, nfg=nfg, zeta=gt["zeta"], J=gt["J"], u1=gt["u1"],
                u2=gt["u2"], seff=gt["seff"], n_fg_nb=n_fg_nb, isum_raw=isum_raw)


# ------------------------------------------------------------------------------------------------------------------
# profiles (`xpg/integrate_kernels.py:154-166`, `:367-380`; `xpg/integrate.py:521-555`)
# ------------------------------------------------------------------------------------------------------------------

def grid_coords(u1, u2, G=PROFILE_GRID):
    """Bilinear cell and weights of normalised coordinates on the profile grid (`:154-166`)."""
    gm1 = F32(G - 1)
    f1 = ((u1 + F32(UMAX)) / F32(2 * UMAX)) * gm1
    f2 = ((u2 + F32(UMAX)) / F32(2 * UMAX)) * gm1
    inside = (f1 >= 0) & (f1 <= gm1) & (f2 >= 0) & (f2 <= gm1)
    top = F32(G - 1 - 1e-4)
    f1 = np.clip(f1, F32(0), top)
    f2 = np.clip(f2, F32(0), top)
    i1 = np.floor(f1).astype(np.int32)
    i2 = np.floor(f2).astype(np.int32)
    t1 = (f1 - i1.astype(F32)).astype(F32)
    t2 = (f2 - i2.astype(F32)).astype(F32)
    return inside, i1, i2, t1, t2


def is_strong_for_profiles(o1):
    """Row selection for profile learning (`xpg/integrate.py:531-533`), in float64 on the float32 outputs."""
    isum = F64(o1["isum"])
    vs = F64(o1["vsum"])
    return bool((isum > 0) and (isum / np.sqrt(max(vs, 1e-6)) > 10.0) and o1["n_over"] == 0
                and F64(o1["frac_rec"]) > 0.95 and o1["n_fg_nb"] == 0 and o1["n_fg_masked"] == 0)


def accumulate(num, den, o1, region, G=PROFILE_GRID):
    """Scatter one strong reflection's normalised projected spot into the float64 grids of its region (`:367-380`)."""
    dens = (o1["img2"] / np.maximum(F32(o1["isum"]), F32(1e-6))) / np.maximum(
        o1["J"] / (F32(o1["seff"]) * F32(o1["seff"])), F32(1e-12))
    inside, i1, i2, t1, t2 = grid_coords(o1["u1"], o1["u2"], G)
    w = (o1["all_valid2"] & inside).astype(F32)
    one = F32(1.0)
    for di, dj, ww in ((0, 0, (one - t1) * (one - t2)), (1, 0, t1 * (one - t2)), (0, 1, (one - t1) * t2),
                       (1, 1, t1 * t2)):
        wv = (w * ww).astype(F32)
        np.add.at(num[region], (i2 + dj, i1 + di), (wv * dens).astype(F32).astype(F64))
        np.add.at(den[region], (i2 + dj, i1 + di), wv.astype(F64))


def finalize_profiles(num, den, G=PROFILE_GRID):
    """Learnt density blended with the Gaussian prior (3 pseudo-counts) and normalised (`xpg/integrate.py:546-555`)."""
    gauss = gaussian_profile(G)
    dens = np.where(den > 0, num / np.maximum(den, 1e-12), 0.0)
    du = (2 * UMAX / (G - 1)) ** 2
    prof = np.empty(num.shape, np.float32)
    for r in range(num.shape[0]):
        emp = np.clip(dens[r], 0, None)
        pr = (den[r] * emp + 3.0 * gauss) / (den[r] + 3.0)
        prof[r] = pr / max(pr.sum() * du, 1e-12)
    return prof


# ------------------------------------------------------------------------------------------------------------------
# pass 2 (`xpg/integrate_kernels.py:278-285`, `:382-483`)
# ------------------------------------------------------------------------------------------------------------------

def profile_plane(prof_r, gt):
    """P2(u) * J / seff^2 per pixel (`:278-285`), (Dy, Dx)."""
    inside, i1, i2, t1, t2 = grid_coords(gt["u1"], gt["u2"], prof_r.shape[-1])
    one = F32(1.0)
    v = ((((one - t1) * (one - t2)) * prof_r[i2, i1] + (t1 * (one - t2)) * prof_r[i2, i1 + 1])
         + ((one - t1) * t2) * prof_r[i2 + 1, i1]) + (t1 * t2) * prof_r[i2 + 1, i1 + 1]
    jn = (gt["J"] / (F32(gt["seff"]) * F32(gt["seff"]))).astype(F32)
    return (np.where(inside, v, F32(0)) * jn).astype(F32)


def pass2(sb, r, nb, det, s0, axis, frames_phi0, osc, sd, sm, gain, prof, bg, nbg, rcw, pix):
    """Profile fit with fixed background and the joint fit of an overlapping partner."""
    sb = f32(sb)
    Dz, Dy, Dx = sb.shape
    gain = F32(gain)
    gt = geometry(det, r, sb.shape, s0, axis, frames_phi0, osc, sd, sm, rcw, pix)
    valid = sb >= 0
    reg = int(r["region"])
    p = (profile_plane(prof[reg], gt)[None] * gt["R"][:, None, None]).astype(F32)
    has_p = bool(r["has_p"] > 0.5)
    if has_p:
        rp = dict(r, S=r["pS"], phi=r["pphi"])
        gtp = geometry(det, rp, sb.shape, s0, axis, frames_phi0, osc, sd, sm, rcw)
        pp = (profile_plane(prof[reg], gtp)[None] * gtp["R"][:, None, None]).astype(F32)
    else:
        pp = np.zeros_like(p)
    nbm = neighbour_mask(gt["x"], gt["y"], gt["zz"], nb, skip_first=has_p)
    c = np.where(valid, sb, F32(0)).astype(F32)
    bref = bkg_ref(det, gt["x"], gt["y"])
    bpix = (F32(bg) * bref).astype(F32)
    net = (c - bpix[None]).astype(F32)
    pmax = p.max()
    ppmax = pp.max()
    use = valid & ~nbm & ((p > F32(0.01) * pmax) | (pp > F32(0.01) * np.maximum(ppmax, F32(1e-12))))
    wp = np.where(use, p, F32(0)).astype(F32)
    wq = np.where(use, pp, F32(0)).astype(F32)
    I = F32(sum32(np.where(use, net, 0)) / np.maximum(sum32(wp + wq), F32(1e-6)))
    hp = F32(1.0 if has_p else 0.0)
    Ip = F32(I * hp)
    wpp = (wp * p).astype(F32)
    wpn = (wp * net).astype(F32)
    wqq = (wq * pp).astype(F32)
    wqn = (wq * net).astype(F32)
    wpq = (wp * pp).astype(F32)
    for _ in range(N_IRLS):
        mu = bpix[None] + np.maximum(I, F32(0)) * p
        if has_p:
            mu = mu + np.maximum(Ip, F32(0)) * pp
        iv = (F32(1.0) / (gain * np.maximum(mu, F32(VAR_FLOOR)))).astype(F32)
        a11 = sum64(wpp * iv)
        b1 = sum64(wpn * iv)
        if has_p:
            a12 = sum64(wpq * iv)
            a22 = sum64(wqq * iv)
            b2 = sum64(wqn * iv)
        else:
            a12, a22, b2 = 0.0, 1.0, 0.0
        det2 = max(a11 * a22 - a12 * a12, 1e-30)
        I = F32((a22 * b1 - a12 * b2) / det2)
        Ip = F32((a11 * b2 - a12 * b1) / det2 * F64(hp))
    # variances, profile correlation and recorded fractions (`:405-429`), float64
    C = sum64((wp * bref[None]).astype(F32) * iv)
    var_b = F64(gain) * max(F64(bg), VAR_FLOOR) / max(F64(nbg), 1.0)
    a11i = a22 / det2
    varI = a11i + (C * a11i) ** 2 * var_b
    iv0 = (F32(1.0) / (gain * np.maximum(bpix, F32(VAR_FLOOR)))).astype(F32)
    a110 = max(sum64(wpp * iv0[None]), 1e-12)
    C0 = sum64((wp * bref[None]).astype(F32) * iv0[None])
    infl = a11i * a11
    var0 = (1.0 / a110 + (C0 / a110) ** 2 * var_b) * max(infl, 1.0)
    nuse = F32(use.sum())
    pm = F32(sum32(wp) / np.maximum(nuse, F32(1)))
    resid = (net - np.maximum(Ip, F32(0)) * pp).astype(F32) if has_p else net
    nm = F32(sum32(np.where(use, resid, 0)) / np.maximum(nuse, F32(1)))
    dp = np.where(use, (p - pm), F32(0)).astype(F32)
    dn = np.where(use, (resid - nm), F32(0)).astype(F32)
    sdd = sum32(dp * dn)
    spp = sum32(dp * dp)
    snn = sum32(dn * dn)
    corr = sdd / np.sqrt(np.maximum(spp * snn, F32(1e-20)))
    p_valid = sum32(np.where(valid & ~nbm, p, F32(0)))
    p_total = sum32(p)
    rho = F32(a12 / np.sqrt(max(a11 * a22, 1e-30))) if has_p else F32(0)
    r2 = (gt["u1"] * gt["u1"] + gt["u2"] * gt["u2"]).astype(F32)
    Rmax = gt["R"].max()
    fgz = gt["R"] >= F32(1e-3) * Rmax + F32(1e-6)
    fgm = (r2 <= F32(FG_R2))[None] & fgz[:, None, None]
    p_fg = sum32(np.where(fgm, p, F32(0))) / np.maximum(p_total, F32(1e-9))
    return dict(iprf=F32(I), vprf=F32(varI), vprf0=F32(var0), corr=F32(corr), p_valid=p_valid, p_total=p_total,
                ipartner=F32(Ip), rho=rho, p_fg=F32(p_fg))
