"""XPG's inner kernel surface on the B200 kernels: `make_kernels(Dz, Dy, Dx, n_regions, G=41)` returns
(pass1, accumulate_profiles, pass2) with the reference's signatures and dict results
(`xpg/integrate_kernels.py:216-485`), for callers that drive the kernels themselves.

Arguments are torch CUDA tensors (numpy arrays are moved to the device): `sb` (N, Dz, Dy, Dx) float32 shoeboxes
(values, -1 masked, -2 overloaded, -3 unrecorded), the `rc` dict (S, phi, ix0, iy0, iz0, fb, region, has_p, pS, pphi
and optionally pxs), the `nb` dict (x, y, z, sx, sz: (N, K)), and `det` from `detector_consts(geometry,
bkg_template)` (XPG's `_detector_consts`). `axis`, `s0`, `frames_phi0`, `osc`, `sd`, `sm`, `gain` and `rcw` as in the
reference. Only Dy == Dx boxes exist in XPG and here.
"""
from __future__ import annotations

import numpy as np
import torch

from . import device as D
from . import native as N

PROFILE_GRID = 41


def detector_consts(g, bkg_template=None, device="cuda"):
    """Device detector description of a geometry (`xpg/integrate_kernels.py:48-65`)."""
    return D.DeviceDetector(g, bkg_template, device)


def _np(v):
    if torch.is_tensor(v):
        return v.detach().cpu().numpy()
    return np.asarray(v)


def _rows(sb, rc, nb, Dz, Dx):
    n = int(sb.shape[0])
    pxs = _np(rc["pxs"]).astype(np.int32) if "pxs" in rc else np.ones(n, np.int32)
    return D.RowSet(S=_np(rc["S"]), phi=_np(rc["phi"]), ix0=_np(rc["ix0"]), iy0=_np(rc["iy0"]), iz0=_np(rc["iz0"]),
                    fb=_np(rc["fb"]), region=_np(rc["region"]), has_p=_np(rc["has_p"]), pS=_np(rc["pS"]),
                    pphi=_np(rc["pphi"]), pxs=pxs, Dz=np.full(n, Dz), bx=np.full(n, Dx),
                    nb={k: _np(nb[k]) for k in ("x", "y", "z", "sx", "sz")}, sb_bias=0.0)


def _block(axis, s0, frames_phi0, osc, sd, sm, gain, rcw):
    b = N.XiBlock()
    b.frames_phi0, b.osc = float(np.float32(frames_phi0)), float(np.float32(osc))
    b.sd, b.sm, b.gain = float(np.float32(sd)), float(np.float32(sm)), float(np.float32(gain))
    rc = torch.as_tensor(_np(rcw).astype(np.float32)).cuda()
    b.rcw = N.ptr(rc)
    a, s = _np(axis).astype(np.float32), _np(s0).astype(np.float32)
    for c in range(3):
        b.axis[c], b.s0[c] = float(a[c]), float(s[c])
    return b, rc


def _sb(sb):
    t = torch.as_tensor(sb) if not torch.is_tensor(sb) else sb
    return t.to("cuda", torch.float32).contiguous().reshape(-1)


def make_kernels(Dz, Dy, Dx, n_regions, G=PROFILE_GRID):
    if Dy != Dx:
        raise ValueError("square boxes only (Dy == Dx)")
    if G != PROFILE_GRID:
        raise ValueError("the kernels use the 41 x 41 profile grid")
    N.require_cuda()

    def pass1(sb, rc, det, axis, s0, frames_phi0, osc, sd, sm, gain, prof, nb, rcw):
        """Background, summation, centroids, 2D projected spot images (`xpg/integrate_kernels.py:287-365`)."""
        rows = _rows(sb, rc, nb, Dz, Dx)
        blk, keep = _block(axis, s0, frames_phi0, osc, sd, sm, gain, rcw)
        arena = _sb(sb)
        out = D.Pass1Buffers(rows)
        D.pass1(det, rows, blk, arena, out)
        D.status()
        t = out.t
        n = rows.n
        res = {k: t[k] for k in D.Pass1Buffers.SCALARS if k not in ("zeta", "seff")}
        res.update({k: t[k] for k in D.Pass1Buffers.COUNTS})
        res["fz"] = t["fz"].view(n, Dz)
        res["img2"] = t["img2"].view(n, Dy, Dx)
        res["all_valid2"] = t["all_valid2"].view(n, Dy, Dx).bool()
        res["zeta"], res["seff"] = t["zeta"], t["seff"]
        res["J"] = t["J"].view(n, Dy, Dx)
        res["u1"] = t["u1"].view(n, Dy, Dx)
        res["u2"] = t["u2"].view(n, Dy, Dx)
        res["_rows"] = rows
        res["_buf"] = out
        return res

    def accumulate_profiles(img2, ok2, J, u1, u2, region, isum, sel, seff):
        """Normalised projected spots scattered into per-region float64 grids (`:367-380`)."""
        n = int(img2.shape[0])
        nbz = {k: np.zeros((n, 1), np.float32) for k in ("x", "y", "z", "sx", "sz")}
        rc = dict(S=np.zeros((n, 3), np.float32), phi=np.zeros(n, np.float32), ix0=np.zeros(n, np.int32),
                  iy0=np.zeros(n, np.int32), iz0=np.zeros(n, np.int32), fb=np.ones(n, np.float32), region=_np(region),
                  has_p=np.zeros(n, np.float32), pS=np.zeros((n, 3), np.float32), pphi=np.zeros(n, np.float32))
        rows = _rows(np.zeros((n, 1, Dy, Dx), np.float32), rc, nbz, 1, Dx)
        buf = D.Pass1Buffers(rows)
        f = lambda v: torch.as_tensor(_np(v)).to("cuda")
        buf.t["img2"].copy_(f(img2).reshape(-1).float())
        buf.t["all_valid2"].copy_(f(ok2).reshape(-1).to(torch.uint8))
        buf.t["J"].copy_(f(J).reshape(-1).float())
        buf.t["u1"].copy_(f(u1).reshape(-1).float())
        buf.t["u2"].copy_(f(u2).reshape(-1).float())
        buf.t["isum"].copy_(f(isum).float())
        buf.t["seff"].copy_(f(seff).float())
        num = torch.zeros((n_regions, G, G), dtype=torch.float64, device="cuda")
        den = torch.zeros_like(num)
        selt = f(sel).to(torch.uint8).contiguous()
        D.accumulate(rows, buf, n_regions, num, den, sel=selt, strong_test=False)
        return num, den

    def pass2(sb, rc, det, axis, s0, frames_phi0, osc, sd, sm, gain, prof, bg, nbm_x, nb, rcw, pix=None):
        """Profile fit with fixed background and the joint fit of overlapping partners (`:382-483`). `pix`: pass 1's
        zeta / J / u1 / u2 / seff of these rows (computed here when absent)."""
        rows = _rows(sb, rc, nb, Dz, Dx)
        arena = _sb(sb)
        if pix is None:
            r1 = pass1(sb, rc, det, axis, s0, frames_phi0, osc, sd, sm, gain, prof, nb, rcw)
            pix = {k: r1[k] for k in ("zeta", "J", "u1", "u2", "seff")}
        buf = D.Pass1Buffers(rows)
        f = lambda v: torch.as_tensor(_np(v)).to("cuda").reshape(-1).float()
        for k in ("zeta", "seff", "J", "u1", "u2"):
            buf.t[k].copy_(f(pix[k]))
        buf.t["bg"].copy_(f(bg))
        buf.t["nbg"].copy_(f(nbm_x))
        blk, keep = _block(axis, s0, frames_phi0, osc, sd, sm, gain, rcw)
        out = D.Pass2Buffers(rows)
        proft = torch.as_tensor(_np(prof).astype(np.float32)).cuda().contiguous()
        D.pass2(det, rows, blk, arena, proft, buf, out)
        D.status()
        return dict(out.t)

    return pass1, accumulate_profiles, pass2
