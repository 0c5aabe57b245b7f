"""Makes forward_terms.npz: the separable profile factors of XPG's forward model (`fraction_terms`,
xpg/forward/model.py:206-280: per reflection R (Dz,) rocking-curve fractions and P (b, b) detector-profile
fractions, one term, or two with the halo) computed by XPG itself for rows of the config-1 fixture's first kernel
chunk (their S, phi, box origins, the chunk's widths and learnt profile), in four variants: parametric Gaussian
profile, learnt profile, learnt profile with the rocking-curve mixture weights, and parametric with a halo.

    XPG_REFERENCE_ROOT=<reference checkout> python tests/golden/make_forward_terms_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

CASE = "config1"
ROWS = 24
VARIANTS = ("gauss", "learnt", "learnt_rcw", "gauss_halo")
HALO = (0.15, 2.5)
UMAX = 0.9 * 5.0


if __name__ == "__main__":
    import torch
    import golden_io as G
    from make_golden import _ref_experiment, _ref_modules
    RI, RK, RGeometry, RCrystal, RExperiment, _ = _ref_modules()
    from xpg.forward import model as RM
    spec = G.case_inputs(CASE)[0]
    exp = _ref_experiment(spec, RGeometry, RCrystal, RExperiment)
    det = RK._detector_consts(exp.geom, None)
    d, rc, nb, o1, o2 = G.chunk(CASE, 0)
    rows = np.flatnonzero(np.asarray(rc["fb"]) == 1)[:ROWS]
    Dz, b = int(d["sb"].shape[1]), int(d["sb"].shape[3])
    t = lambda a, dt=torch.float32: torch.as_tensor(np.asarray(a), dtype=dt)
    save = dict(rows=rows, Dz=np.int64(Dz), b=np.int64(b), umax=np.float64(UMAX), halo=np.array(HALO),
                frames_phi0=np.float64(d["frames_phi0"]), osc=np.float64(d["osc"]), sd=np.float64(d["sd"]),
                sm=np.float64(d["sm"]), s0=np.asarray(d["s0"], np.float64), axis=np.asarray(d["axis"], np.float64),
                rcw=np.asarray(d["rcw"], np.float32), prof=np.asarray(d["prof"], np.float32),
                S=np.asarray(rc["S"][rows], np.float32), phi=np.asarray(rc["phi"][rows], np.float32),
                ix0=np.asarray(rc["ix0"][rows], np.int64), iy0=np.asarray(rc["iy0"][rows], np.int64),
                iz0=np.asarray(rc["iz0"][rows], np.int64), region=np.asarray(rc["region"][rows], np.int64))
    for v in VARIANTS:
        prof = t(save["prof"]) if v.startswith("learnt") else None
        rcw = t(save["rcw"]) if v == "learnt_rcw" else None
        halo = HALO if v.endswith("halo") else None
        terms = RM.fraction_terms(det, t(save["axis"]), t(save["s0"]), float(save["frames_phi0"]),
                                  float(save["osc"]), float(save["sd"]), float(save["sm"]), t(save["S"]),
                                  t(save["phi"]), t(save["ix0"], torch.int64), t(save["iy0"], torch.int64),
                                  t(save["iz0"], torch.int64), Dz, b, prof=prof, region=t(save["region"], torch.int64),
                                  umax=UMAX, halo=halo, rcw=rcw)
        for k, (R, P) in enumerate(terms):
            save[f"{v}_R{k}"] = R.numpy().astype(np.float32)
            save[f"{v}_P{k}"] = P.numpy().astype(np.float32)
        save[f"{v}_n_terms"] = np.int64(len(terms))
    np.savez_compressed(HERE / "forward_terms.npz", **save)
    print((HERE / "forward_terms.npz").stat().st_size)
