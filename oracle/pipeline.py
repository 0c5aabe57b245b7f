"""CPU restatement of the per-reflection integration pipeline (frame preparation, gather, pass 1, pass 2) for a set
of rows of a shoebox plan: TEST INFRASTRUCTURE and the timed CPU baseline of bench.py (see oracle/__init__.py).

It follows XPG's CPU path for the same rows (`xpg/integrate.py:648-787` for the frames, then
`xpg/integrate_kernels.py:287-483` per reflection) with the block constants given (no profile learning: the
Gaussian prior profile, `xpg/integrate.py:546-555` with empty grids)."""
from __future__ import annotations

import numpy as np

from . import gather as OG
from . import kernels as OK


def prepared_frames(raw_frames, first_fi, overload, pxs_set, mask=None):
    """{s: {fi: prepared frame at super-pixel scale s}} of consecutive raw uint32 frames starting at first_fi."""
    out = {s: {} for s in pxs_set}
    for w, raw in enumerate(raw_frames):
        pf = OG.prepare_frame(raw, overload, 0, mask)
        for s in pxs_set:
            out[s][first_fi + w] = pf if s == 1 else OG.superpixel_frame(pf, s)
    return out


def row_payload(plan, rows):
    """Self-contained per-row inputs of plan rows (picklable: what a worker process needs)."""
    out = []
    for j in rows:
        pj = plan.partner[j]
        r = dict(S=plan.refl["S"][j].astype(np.float32), phi=np.float32(np.radians(plan.refl["phi"][j])),
                 ix0=int(plan.ix0[j]), iy0=int(plan.iy0[j]), iz0=int(plan.iz0[j]), fb=np.float32(plan.fb[j]),
                 region=int(plan.region[j]), has_p=np.float32(plan.has_partner[j]),
                 pS=plan.refl["S"][pj].astype(np.float32), pphi=np.float32(np.radians(plan.refl["phi"][pj])),
                 pxs=int(plan.pxs[j]), Dz=int(plan.Dz[j]), bx=int(plan.bx[j]), fbi=int(plan.fb[j]))
        nb = {k: v[j] for k, v in plan.nb.items()}
        out.append((r, nb))
    return out


def integrate_rows(prepared, read_fi, payload, det, s0, axis, frames_phi0, osc, sd, sm, gain, rcw, prof,
                   origin=(0, 0)):
    """pass-1 and pass-2 outputs of rows (row_payload) from prepared frames (dict per super-pixel scale); `origin`:
    array indices (y, x) of the prepared frames' first pixel when they are crops of the detector."""
    res = []
    y0, x0 = origin
    for r, nb in payload:
        sb = OG.gather_shoebox(prepared[r["pxs"]], read_fi, r["iz0"], r["fbi"], r["Dz"], r["bx"], r["iy0"] - y0,
                               r["ix0"] - x0)
        o1 = OK.pass1(sb, r, nb, det, s0, axis, frames_phi0, osc, sd, sm, gain, rcw)
        pix = dict(zeta=o1["zeta"], J=o1["J"], u1=o1["u1"], u2=o1["u2"], seff=o1["seff"])
        o2 = OK.pass2(sb, r, nb, det, s0, axis, frames_phi0, osc, sd, sm, gain, prof, o1["bg"], o1["nbg"], rcw, pix)
        res.append((o1, o2))
    return res
