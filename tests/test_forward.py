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
