"""The forward-model likelihood passes' CPU restatement (oracle/forward.py) against XPG's own passes on the same
inputs (tests/golden/forward.npz: `WindowModel.mu`, `grad_ratio`, `grad_newton`, xpg/forward/model.py:476-577)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

from oracle import forward as OF

GOLD = Path(__file__).resolve().parent / "golden" / "forward.npz"
RTOL = 1e-5          # float32 sums in another order


def cases():
    z = np.load(GOLD)
    out = []
    for k in range(int(z["n_cases"])):
        c = {key[len(f"c{k}_"):]: z[key] for key in z.files if key.startswith(f"c{k}_")}
        c["groups"] = [dict(R=c[f"g{g}_R"], P=c[f"g{g}_P"], iz0=c[f"g{g}_iz0"], iy0=c[f"g{g}_iy0"],
                            ix0=c[f"g{g}_ix0"], rows=c[f"g{g}_rows"]) for g in range(int(c["n_groups"]))]
        out.append(c)
    return out


def close(a, b, scale):
    return np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) <= RTOL * scale


def test_oracle_passes_match_xpg():
    for c in cases():
        beta = c["beta"] if c["beta"].size else None
        mu = OF.scatter(c["B"], c["groups"], c["I"], beta, c["win"])
        assert close(mu, c["xpg_mu"], np.maximum(np.abs(mu), 1.0)).all()
        n = int(c["n"])
        gr, _ = OF.gather(c["groups"], c["win"], n, c["A"], c["M"], c["NS"], 0)
        gn, fd = OF.gather(c["groups"], c["win"], n, None, c["M"], c["NS"], 1)
        for ours, xpg in ((gr, c["xpg_grad_ratio"]), (gn, c["xpg_grad_newton"]), (fd, c["xpg_fisher_diag"])):
            assert close(ours, xpg, np.maximum(np.abs(ours), 1e-3)).all()


def test_cases_reach_every_edge():
    """The fixtures hold boxes outside the window in every direction, overlapping boxes and invalid voxels."""
    for c in cases():
        f0, f1, y0, ny, x0, nx = c["win"]
        edge = np.zeros(6, bool)
        for g in c["groups"]:
            Dz, b = g["R"].shape[2], g["P"].shape[-1]
            edge |= [(g["iz0"] < f0).any(), (g["iz0"] + Dz > f1).any(), (g["iy0"] < y0).any(),
                     (g["iy0"] + b > y0 + ny).any(), (g["ix0"] < x0).any(), (g["ix0"] + b > x0 + nx).any()]
        assert edge.all()
        assert (c["NS"] < 0).any()


def test_oracle_fraction_terms_match_xpg():
    """The separable factors (`fraction_terms`, xpg/forward/model.py:206-280) against XPG's own on rows of the
    config-1 fixture (tests/golden/forward_terms.npz): parametric and learnt profiles, the rocking-curve mixture, the
    halo's second term; within 1e-6 of each reflection's largest factor."""
    import golden_io as G
    from oracle import kernels as OK
    z = np.load(Path(__file__).resolve().parent / "golden" / "forward_terms.npz")
    spec = G.case_inputs("config1")[0]
    det = OK.detector_consts(spec.geometry(), None)
    Dz, b = int(z["Dz"]), int(z["b"])
    worst = 0.0
    for v in ("gauss", "learnt", "learnt_rcw", "gauss_halo"):
        terms = OF.fraction_terms(det, z["S"], z["phi"], z["ix0"], z["iy0"], z["iz0"], Dz, b, z["s0"], z["axis"],
                                  float(z["frames_phi0"]), float(z["osc"]), float(z["sd"]), float(z["sm"]),
                                  prof=z["prof"] if v.startswith("learnt") else None, region=z["region"],
                                  umax=float(z["umax"]), halo=tuple(z["halo"]) if v.endswith("halo") else None,
                                  rcw=z["rcw"] if v == "learnt_rcw" else None)
        assert len(terms) == int(z[f"{v}_n_terms"])
        for k, (R, P) in enumerate(terms):
            for ours, xpg in ((R, z[f"{v}_R{k}"]), (P, z[f"{v}_P{k}"])):
                scale = np.abs(xpg).max(axis=tuple(range(1, xpg.ndim)), keepdims=True)
                err = np.abs(ours.astype(np.float64) - xpg) / np.maximum(scale, 1e-30)
                worst = max(worst, float(err.max()))
                assert err.max() <= 1e-6, (v, k, float(err.max()))      # float32 rounding (measured 4e-7)
    assert worst < 1e-6
