"""All-float64 restatement of the per-reflection integration kernels: TEST INFRASTRUCTURE (see oracle/__init__.py).

The same algorithm as `oracle/kernels.py` (`xpg/integrate_kernels.py:68-483`: pixel geometry, pass 1, profile
accumulation and finalisation, pass 2), with every operation in float64: detector constants, the Kabsch mapping, the
pixel area, the rocking curve, every mask test, sum and fit. It is the reference the precision report measures the
float32 device path against (error of I and sigma by resolution shell and I/sigma bin). Masks are decided in float64
here, so a voxel on a mask boundary may fall on the other side than in float32: that is part of the measured error.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

F = np.float64
N_FG = 3.0
FG_R2 = 9.0
BG_R2 = 12.25
G = 41
UMAX = 4.5
N_IRLS = 6
VAR_FLOOR = 1e-3
RC_C = np.linspace(-3.5, 3.5, 21)
RC_W = 0.25


def detector(g, bkg_template=None):
    """Detector constants in float64 (`xpg/integrate_kernels.py:48-65`)."""
    P0, Bx, By = (np.asarray(a, F).reshape(-1, 3) for a in g.panels())
    U1, U2 = Bx / g.qx, By / g.qy
    segmap = g.segmap() if getattr(g, "segmented", False) else None
    geo = getattr(g, "geo_corr", None)
    return dict(orgx=F(g.orgx), orgy=F(g.orgy), qx=F(g.qx), qy=F(g.qy), P0=P0, Bx=Bx, By=By, U1=U1, U2=U2,
                UN=np.cross(U1, U2), segmap=segmap, gx=None if geo is None else np.asarray(geo[0], F),
                gy=None if geo is None else np.asarray(geo[1], F), wl=F(g.wavelength),
                tsens=F(max(g.sensor_thickness, 1e-6)), mu=F(max(g.mu, 1e-6)), plx=bool(g.has_parallax),
                bkg=None if bkg_template is None else np.asarray(bkg_template, F))


def _bilinear_table(tab, x, y):
    ny, nx = tab.shape
    fx = np.clip(x - 1.0, 0.0, nx - 1.000001)
    fy = np.clip(y - 1.0, 0.0, ny - 1.000001)
    ix, iy = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
    ix1, iy1 = np.minimum(ix + 1, nx - 1), np.minimum(iy + 1, ny - 1)
    tx, ty = fx - ix, fy - iy
    return (tab[iy, ix] * (1 - tx) * (1 - ty) + tab[iy, ix1] * tx * (1 - ty) + tab[iy1, ix] * (1 - tx) * ty
            + tab[iy1, ix1] * tx * ty)


def pixel_S(det, x, y):
    """Diffracted wave vector of detector points (`xpg/integrate_kernels.py:78-105`)."""
    if det["segmap"] is None:
        k = np.zeros(x.shape, np.int64)
    else:
        sm = det["segmap"]
        ix = np.clip(np.floor(x - 0.5).astype(np.int64), 0, sm.shape[1] - 1)
        iy = np.clip(np.floor(y - 0.5).astype(np.int64), 0, sm.shape[0] - 1)
        k = np.maximum(sm[iy, ix], 0).astype(np.int64)
    P0, Bx, By, U1, U2, UN = (det[n][k] for n in ("P0", "Bx", "By", "U1", "U2", "UN"))
    if det["gx"] is None:
        xc, yc = x, y
    else:
        xc, yc = x + _bilinear_table(det["gx"], x, y), y + _bilinear_table(det["gy"], x, y)

    def plane(xx, yy):
        return P0 + (xx - det["orgx"])[..., None] * Bx + (yy - det["orgy"])[..., None] * By
    X = plane(xc, yc)
    for _ in range(2 if det["plx"] else 0):
        e = X / np.linalg.norm(X, axis=-1, keepdims=True)
        cosa = np.clip(np.sum(e * UN, -1), 1e-3, 1.0)
        L = det["tsens"] / cosa
        muL = det["mu"] * L
        lbar = 1.0 / det["mu"] - L * np.exp(-muL) / np.maximum(-np.expm1(-muL), 1e-12)
        X = plane(xc - lbar * np.sum(e * U1, -1) / det["qx"], yc - lbar * np.sum(e * U2, -1) / det["qy"])
    return X / (np.linalg.norm(X, axis=-1, keepdims=True) * det["wl"])


def bkg_ref(det, x, y):
    if det["bkg"] is None:
        return np.ones((y.size, x.size), F)
    ny, nx = det["bkg"].shape
    ix = np.clip(np.rint(x - 1.0).astype(np.int64), 0, nx - 1)
    iy = np.clip(np.rint(y - 1.0).astype(np.int64), 0, ny - 1)
    return det["bkg"][iy[:, None], ix[None, :]]


def _grad(f, axis):
    g = np.empty_like(f)
    sl = lambda i: tuple(slice(None) if a != axis else i for a in range(f.ndim))
    g[sl(slice(1, -1))] = (f[sl(slice(2, None))] - f[sl(slice(None, -2))]) / 2.0
    g[sl(0)] = -1.5 * f[sl(0)] + 2.0 * f[sl(1)] - 0.5 * f[sl(2)]
    g[sl(-1)] = 0.5 * f[sl(-3)] - 2.0 * f[sl(-2)] + 1.5 * f[sl(-1)]
    return g


def geometry(det, r, shape, s0, axis, frames_phi0, osc, sd, sm, rcw):
    """Per-reflection mapping (`xpg/integrate_kernels.py:219-276`) in float64."""
    Dz, Dy, Dx = shape
    s = F(r.get("pxs", 1))
    x = (F(r["ix0"]) + np.arange(Dx)) * s + (s - 1) * 0.5 + 1.0
    y = (F(r["iy0"]) + np.arange(Dy)) * s + (s - 1) * 0.5 + 1.0
    fb = F(r["fb"])
    zz = F(r["iz0"]) + fb * (np.arange(Dz) + 0.5)
    S = np.asarray(r["S"], F)
    c1 = np.cross(S, s0)
    e1 = c1 / np.linalg.norm(c1)
    c2 = np.cross(S, e1)
    e2 = c2 / np.linalg.norm(c2)
    zeta = F(e1 @ axis)
    X, Y = np.meshgrid(x, y)
    d = pixel_S(det, X, Y) - S
    eps1, eps2 = (d @ e1) / np.linalg.norm(S), (d @ e2) / np.linalg.norm(S)
    J = np.abs(_grad(eps1, 1) * _grad(eps2, 0) - _grad(eps2, 1) * _grad(eps1, 0))
    seff = sd * np.sqrt(1.0 + (np.sqrt(J[Dy // 2, Dx // 2]) / sd) ** 2 / 12.0)
    k = F(r["iz0"]) + fb * np.arange(Dz)
    plo = frames_phi0 + osc * k
    phi_ = plo + osc * fb
    lo, hi = np.minimum(plo, phi_), np.maximum(plo, phi_)
    sw_s = sm / max(abs(zeta), 1e-3)
    sw = sw_s * RC_W * np.sqrt(2.0)
    phi = F(r["phi"])
    a = (hi[:, None] - phi - RC_C * sw_s) / sw
    b = (lo[:, None] - phi - RC_C * sw_s) / sw
    R = (np.asarray(rcw, F) * 0.5 * (erf(a) - erf(b))).sum(1)
    return dict(x=x, y=y, zz=zz, u1=eps1 / seff, u2=eps2 / seff, J=J, R=R, zeta=zeta, phi_c=0.5 * (lo + hi),
                seff=seff)


def neighbour_mask(x, y, zz, nb, skip_first=False):
    m = np.zeros((zz.size, y.size, x.size), bool)
    for k in range(len(nb["x"])):
        if k == 0 and skip_first:
            continue
        sx, sz = F(nb["sx"][k]), F(nb["sz"][k])
        dx, dy, dz = (x - F(nb["x"][k])) / sx, (y - F(nb["y"][k])) / sx, (zz - F(nb["z"][k])) / sz
        m |= (dx[None, None, :] ** 2 + dy[None, :, None] ** 2 + dz[:, None, None] ** 2) < 1.0
    return m


def pass1(sb, r, nb, det, s0, axis, frames_phi0, osc, sd, sm, gain, rcw):
    """`xpg/integrate_kernels.py:287-365` in float64: background, summation, centroid, moments, projected spot."""
    sb = np.asarray(sb, F)
    gt = geometry(det, r, sb.shape, s0, axis, frames_phi0, osc, sd, sm, rcw)
    valid, recorded, over = sb >= 0, sb > -2.5, sb == -2
    r2 = gt["u1"] ** 2 + gt["u2"] ** 2
    fg2 = r2 <= FG_R2
    fgz = gt["R"] >= 1e-3 * gt["R"].max() + 1e-6
    fg = fg2[None] & fgz[:, None, None]
    nbm = neighbour_mask(gt["x"], gt["y"], gt["zz"], nb)
    bgm = valid & ~fg & ~nbm & (r2 >= BG_R2)[None]
    c = np.where(valid, sb, 0.0)
    bref = bkg_ref(det, gt["x"], gt["y"])
    w = bgm
    b = np.where(w, c, 0).sum() / max(np.where(w, bref[None], 0).sum(), 1e-6)
    for _ in range(4):
        bp = b * bref
        thr = bp + 3.0 * np.sqrt(gain * np.maximum(bp, 0.5)) + 1.0
        w = bgm & (c <= thr[None])
        b = np.where(w, c, 0).sum() / max(np.where(w, bref[None], 0).sum(), 1e-6)
    nbg = np.where(w, bref[None], 0).sum()
    fgv = fg & valid & ~nbm
    bpix = b * bref
    net = c - bpix[None]
    sfb = np.where(fgv, bref[None], 0).sum()
    tail = sfb * sfb * gain * max(b, VAR_FLOOR) / max(nbg, 1.0)
    isum = np.where(fgv, net, 0).sum()
    vsum = gain * np.where(fgv, c, 0).sum() + tail
    clean = valid & ~nbm
    img2 = np.where(fgz[:, None, None] & clean, net, 0).sum(0)
    all_valid2 = (clean | ~fgz[:, None, None]).all(0)
    fz = np.where(fg2[None] & valid & ~nbm, net, 0).sum((1, 2))
    return dict(bg=b, nbg=nbg, isum=isum, vsum=vsum, img2=img2, all_valid2=all_valid2, fz=fz,
                n_over=int((over & fg).sum()), n_fg_masked=int((fg & ~valid & recorded).sum()),
                n_fg_nb=int((fg & nbm).sum()), frac_rec=np.where(recorded.any((1, 2)), gt["R"], 0).sum(),
                isum_raw=int(np.where(fgv, c, 0).sum()), gt=gt)


def strong_for_profiles(o1):
    """`xpg/integrate.py:531-533`."""
    return bool(o1["isum"] > 0 and o1["isum"] / np.sqrt(max(o1["vsum"], 1e-6)) > 10.0 and o1["n_over"] == 0
                and o1["frac_rec"] > 0.95 and o1["n_fg_nb"] == 0 and o1["n_fg_masked"] == 0)


def _cell(u1, u2):
    f1 = (u1 + UMAX) / (2 * UMAX) * (G - 1)
    f2 = (u2 + UMAX) / (2 * UMAX) * (G - 1)
    inside = (f1 >= 0) & (f1 <= G - 1) & (f2 >= 0) & (f2 <= G - 1)
    f1, f2 = np.clip(f1, 0, G - 1 - 1e-4), np.clip(f2, 0, G - 1 - 1e-4)
    i1, i2 = np.floor(f1).astype(np.int64), np.floor(f2).astype(np.int64)
    return inside, i1, i2, f1 - i1, f2 - i2


def accumulate(num, den, o1, region):
    """`xpg/integrate_kernels.py:367-380` in float64."""
    gt = o1["gt"]
    dens = (o1["img2"] / max(o1["isum"], 1e-6)) / np.maximum(gt["J"] / gt["seff"] ** 2, 1e-12)
    inside, i1, i2, t1, t2 = _cell(gt["u1"], gt["u2"])
    w = (o1["all_valid2"] & inside).astype(F)
    for di, dj, ww in ((0, 0, (1 - t1) * (1 - t2)), (1, 0, t1 * (1 - t2)), (0, 1, (1 - t1) * t2), (1, 1, t1 * t2)):
        np.add.at(num[region], (i2 + dj, i1 + di), w * ww * dens)
        np.add.at(den[region], (i2 + dj, i1 + di), w * ww)


def finalize(num, den):
    """`xpg/integrate.py:546-555` in float64."""
    u = np.linspace(-UMAX, UMAX, G)
    U1, U2 = np.meshgrid(u, u)
    gauss = np.exp(-0.5 * (U1 ** 2 + U2 ** 2)) / (2 * np.pi)
    du = (2 * UMAX / (G - 1)) ** 2
    out = np.empty(num.shape)
    for r in range(num.shape[0]):
        emp = np.clip(np.where(den[r] > 0, num[r] / np.maximum(den[r], 1e-12), 0.0), 0, None)
        pr = (den[r] * emp + 3.0 * gauss) / (den[r] + 3.0)
        out[r] = pr / max(pr.sum() * du, 1e-12)
    return out


def _plane(prof_r, gt):
    inside, i1, i2, t1, t2 = _cell(gt["u1"], gt["u2"])
    v = ((1 - t1) * (1 - t2) * prof_r[i2, i1] + t1 * (1 - t2) * prof_r[i2, i1 + 1] + (1 - t1) * t2 * prof_r[i2 + 1, i1]
         + t1 * t2 * prof_r[i2 + 1, i1 + 1])
    return np.where(inside, v, 0.0) * gt["J"] / gt["seff"] ** 2


def pass2(sb, r, nb, det, s0, axis, frames_phi0, osc, sd, sm, gain, prof, o1, rcw):
    """`xpg/integrate_kernels.py:382-483` in float64 (pass 1's background and the same sigma_D)."""
    sb = np.asarray(sb, F)
    gt = geometry(det, r, sb.shape, s0, axis, frames_phi0, osc, sd, sm, rcw)
    valid = sb >= 0
    reg = int(r["region"])
    p = _plane(prof[reg], gt)[None] * gt["R"][:, None, None]
    has_p = bool(r["has_p"] > 0.5)
    if has_p:
        gtp = geometry(det, dict(r, S=r["pS"], phi=r["pphi"]), sb.shape, s0, axis, frames_phi0, osc, sd, sm, rcw)
        pp = _plane(prof[reg], gtp)[None] * gtp["R"][:, None, None]
    else:
        pp = np.zeros_like(p)
    nbm = neighbour_mask(gt["x"], gt["y"], gt["zz"], nb, skip_first=has_p)
    c = np.where(valid, sb, 0.0)
    bref = bkg_ref(det, gt["x"], gt["y"])
    bg, nbg = o1["bg"], o1["nbg"]
    bpix = bg * bref
    net = c - bpix[None]
    use = valid & ~nbm & ((p > 0.01 * p.max()) | (pp > 0.01 * max(pp.max(), 1e-12)))
    wp, wq = np.where(use, p, 0), np.where(use, pp, 0)
    I = np.where(use, net, 0).sum() / max((wp + wq).sum(), 1e-6)
    Ip = I * (1.0 if has_p else 0.0)
    for _ in range(N_IRLS):
        mu = bpix[None] + max(I, 0.0) * p + (max(Ip, 0.0) * pp if has_p else 0.0)
        iv = 1.0 / (gain * np.maximum(mu, VAR_FLOOR))
        a11, b1 = (wp * p * iv).sum(), (wp * net * iv).sum()
        if has_p:
            a12, a22, b2 = (wp * pp * iv).sum(), (wq * pp * iv).sum(), (wq * net * iv).sum()
        else:
            a12, a22, b2 = 0.0, 1.0, 0.0
        det2 = max(a11 * a22 - a12 * a12, 1e-30)
        I = (a22 * b1 - a12 * b2) / det2
        Ip = (a11 * b2 - a12 * b1) / det2 * (1.0 if has_p else 0.0)
    C = (wp * bref[None] * iv).sum()
    var_b = gain * max(bg, VAR_FLOOR) / max(nbg, 1.0)
    a11i = a22 / det2
    varI = a11i + (C * a11i) ** 2 * var_b
    return dict(iprf=I, vprf=varI, p_valid=np.where(valid & ~nbm, p, 0).sum(), p_total=p.sum())
