"""Precision of the device path against the all-float64 restatement (oracle/fp64.py) on the precision sweep: config 1's
geometry (1030 x 1065 px, 100 frames of 0.1 deg, P4_32_12 79/79/38 A) with 5% weak reflections (mean 2 photons)
and 2% of the boxes more than 40% masked by dead rectangles.

The sweep is integrated by the drop-in `integrate()` on the GPU (float32 voxel arithmetic, float64 accumulation and
fit). The float64 restatement then integrates every reflection again from the same frames: pass 1 in float64, the
profiles learnt in float64 from its own strong rows, pass 2 in float64 with those profiles and the device run's
adapted widths (the width adaptation is float64 in both). The errors of the summation intensity, the profile-fitted
intensity and its sigma are tabulated by resolution shell and by I/sigma bin: the median and the 99th percentile
and maximum of |dI| / max(|I|, sigma) (the tolerance's measure) and of |d sigma| / sigma.

    python tests/precision_report.py > profiles/precision_config3.md      (on a machine with a B200)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

I_SIG_EDGES = (-np.inf, 1.0, 3.0, 10.0, 30.0, 100.0, np.inf)
N_SHELLS = 6


def run(device="cuda"):
    """Per-reflection results of the device run and of the float64 restatement: dict of arrays."""
    from oracle import fp64 as O
    from oracle import gather as OG
    from xpg_b200 import synth
    from xpg_b200.frames import U32Frames
    from xpg_b200.integrate import integrate
    from xpg_b200.plan import IntegrationModel, plan_integration
    spec = synth.config3()
    exp = spec.experiment()
    g = exp.geom
    edges = spec.block_edges()
    model = IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m)
    dmin = spec.resolution_limit()
    raw = synth.render_frames(spec)
    res = integrate(U32Frames(raw, first=1, overload=spec.overload), [exp] * (len(edges) - 1), edges, model, dmin,
                    frames=(1, spec.nframes), verbose=False, n_regions_xy=spec.n_regions_xy)
    p = plan_integration([exp] * (len(edges) - 1), edges, model, dmin, 1e9, (1, spec.nframes), 0.05,
                         spec.n_regions_xy, True, True)
    prep = {fi: OG.prepare_frame(raw[fi], spec.overload) for fi in range(spec.nframes)}
    det = O.detector(g)
    s0, axis = np.asarray(g.s0, float), np.asarray(g.axis, float)
    phi0, osc = float(np.float32(np.radians(g.z_to_phi(0.0)))), float(np.float32(np.radians(g.osc)))
    out = {k: np.full(p.n, np.nan) for k in ("isum", "iprf", "vprf", "p_valid", "p_total")}
    for b, rows in enumerate(p.blocks_refl):
        if not rows.size:
            continue
        (sd1, sm1, rcw1), (sd2, sm2, rcw2) = res.block_widths[b]["pass1"], res.block_widths[b]["pass2"]
        num = np.zeros((p.nreg, O.G, O.G))
        den = np.zeros_like(num)
        keep = {}
        for j in rows:
            r = _row(p, j)
            sb = OG.gather_shoebox(prep, range(spec.nframes), r["iz0"], r["fbi"], r["Dz"], r["bx"], r["iy0"],
                                   r["ix0"])
            nb = {k: v[j] for k, v in p.nb.items()}
            o1 = O.pass1(sb, r, nb, det, s0, axis, phi0, osc, sd1, sm1, model.gain, rcw1)
            if O.strong_for_profiles(o1):
                O.accumulate(num, den, o1, r["region"])
            keep[j] = (r, nb, sb, o1)
            out["isum"][j] = o1["isum"]
        prof = O.finalize(num, den)
        for j, (r, nb, sb, o1) in keep.items():
            o2 = O.pass2(sb, r, nb, det, s0, axis, phi0, osc, sd2, sm2, model.gain, prof, o1, rcw2)
            for k in ("iprf", "vprf", "p_valid", "p_total"):
                out[k][j] = o2[k]
    d = 1.0 / np.linalg.norm(p.refl["S"] - np.asarray(g.s0, float), axis=1)     # resolution of each reflection
    return dict(d=d, gpu={k: np.asarray(res.refl[k], float) for k in ("isum", "vsum", "iprf", "vprf", "p_valid",
                                                                      "p_total")}, f64=out,
                weak=None, n=p.n)


def _row(p, j):
    pj = int(p.partner[j])
    return dict(S=p.refl["S"][j], phi=np.radians(p.refl["phi"][j]), ix0=int(p.ix0[j]), iy0=int(p.iy0[j]),
                iz0=int(p.iz0[j]), fb=float(p.fb[j]), fbi=int(p.fb[j]), region=int(p.region[j]),
                has_p=float(p.has_partner[j]), pS=p.refl["S"][pj], pphi=np.radians(p.refl["phi"][pj]),
                pxs=int(p.pxs[j]), Dz=int(p.Dz[j]), bx=int(p.bx[j]))


def errors(r):
    """Per-reflection error measures (NaN where a reflection has no fit)."""
    g, f = r["gpu"], r["f64"]
    sig = np.sqrt(np.maximum(f["vprf"], 1e-12))
    sig_s = np.sqrt(np.maximum(g["vsum"], 1e-12))
    return dict(isum=np.abs(g["isum"] - f["isum"]) / np.maximum(np.abs(f["isum"]), sig_s),
                iprf=np.abs(g["iprf"] - f["iprf"]) / np.maximum(np.abs(f["iprf"]), sig),
                sprf=np.abs(np.sqrt(np.maximum(g["vprf"], 0)) - sig) / sig,
                isig=f["iprf"] / sig, fitted=f["p_valid"] >= 0.01 * f["p_total"])


def _stats(e):
    e = e[np.isfinite(e)]
    if not e.size:
        return "-", "-", "-"
    return f"{np.median(e):.1e}", f"{np.percentile(e, 99):.1e}", f"{e.max():.1e}"


def table(r):
    """Markdown tables of the errors by resolution shell and by I/sigma bin (rows with >= 1% of the profile on valid
    pixels; the others are counted separately)."""
    e = errors(r)
    ok = e["fitted"] & np.isfinite(e["iprf"])
    lines = [f"Reflections: {r['n']}, with a profile fit on >= 1% valid profile: {int(ok.sum())}; "
             f"the rest ({int((~ok).sum())}) are extrapolations from a handful of pixels (PEAK < 1%).", ""]
    head = ("| {} | n | I_sum median / p99 / max | I_prf median / p99 / max | sigma_prf median / p99 / max |\n"
            "|---|---|---|---|---|")
    d = r["d"]
    inv = 1.0 / d[ok] ** 3
    qs = np.quantile(inv, np.linspace(0, 1, N_SHELLS + 1))
    shell = np.clip(np.searchsorted(qs, 1.0 / d ** 3, side="right") - 1, 0, N_SHELLS - 1)
    lines.append(head.format("resolution shell (A)"))
    for s in range(N_SHELLS):
        m = ok & (shell == s)
        lo, hi = (1.0 / qs[s + 1]) ** (1 / 3), (1.0 / qs[s]) ** (1 / 3)
        lines.append(f"| {hi:.2f}-{lo:.2f} | {int(m.sum())} | " + " | ".join(
            " / ".join(_stats(e[k][m])) for k in ("isum", "iprf", "sprf")) + " |")
    lines += ["", head.format("I/sigma")]
    for a, b in zip(I_SIG_EDGES[:-1], I_SIG_EDGES[1:]):
        m = ok & (e["isig"] >= a) & (e["isig"] < b)
        lines.append(f"| {a:g} to {b:g} | {int(m.sum())} | " + " | ".join(
            " / ".join(_stats(e[k][m])) for k in ("isum", "iprf", "sprf")) + " |")
    return "\n".join(lines)


if __name__ == "__main__":
    r = run()
    print("# Precision of the device path against the all-float64 restatement (precision sweep)\n")
    print("Command: `python tests/precision_report.py` on one B200. Errors: |d| / max(|value|, sigma) for "
          "intensities, |d sigma| / sigma for sigma.\n")
    print(table(r))
