"""Makes forward.npz: inputs and outputs of XPG's forward-model likelihood passes run by XPG itself (the eager
`WindowModel.mu`, `grad_ratio` and `grad_newton`, xpg/forward/model.py:476-577, which the fused Triton kernels of
xpg/forward/kernels.py:34-134 replace on CUDA) on seeded synthetic separable profile factors. A WindowModel is made
without its planning: each case sets the window and the chunks' factors (R, P), box origins and rows directly, the
state the passes read.

Cases: one and two separable terms; boxes partly outside the window in frames, rows and columns; overlapping boxes
(several reflections adding to a voxel); with and without the per-reflection flat level beta; counts with invalid
(-1) voxels.

    XPG_REFERENCE_ROOT=<reference checkout> python tests/golden/make_forward_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

# (window f0, f1, y0, ny, x0, nx), groups [(n, Dz, b)], terms, with beta
CASES = [
    ((3, 13, 10, 30, 20, 36), [(30, 5, 7), (12, 9, 11)], 1, True),
    ((0, 9, 0, 25, 0, 29), [(25, 3, 9), (8, 5, 13), (6, 9, 5)], 2, False),
    ((5, 22, 7, 40, 11, 44), [(60, 9, 9), (10, 17, 17)], 2, True),
]


def case_inputs(k):
    (f0, f1, y0, ny, x0, nx), groups, T, with_beta = CASES[k]
    rng = np.random.default_rng(40 + k)
    n = sum(g[0] for g in groups)
    out = dict(win=np.array([f0, f1, y0, ny, x0, nx], np.int64), T=np.int64(T), n=np.int64(n))
    row0 = 0
    for gi, (m, Dz, b) in enumerate(groups):
        R = rng.uniform(0.0, 1.0, (T, m, Dz)).astype(np.float32)
        P = rng.uniform(0.0, 0.02, (T, m, b, b)).astype(np.float32)
        # box origins spread over the window and a margin around it (partly outside in every direction)
        iz0 = rng.integers(f0 - Dz + 1, f1, m).astype(np.int64)
        iy0 = rng.integers(y0 - b + 1, y0 + ny, m).astype(np.int64)
        ix0 = rng.integers(x0 - b + 1, x0 + nx, m).astype(np.int64)
        out.update({f"g{gi}_R": R, f"g{gi}_P": P, f"g{gi}_iz0": iz0, f"g{gi}_iy0": iy0, f"g{gi}_ix0": ix0,
                    f"g{gi}_rows": np.arange(row0, row0 + m, dtype=np.int64), f"g{gi}_shape": np.array([m, Dz, b])})
        row0 += m
    out["n_groups"] = np.int64(len(groups))
    nv = (f1 - f0) * ny * nx
    out["I"] = rng.uniform(-5.0, 400.0, n).astype(np.float32)
    out["beta"] = rng.uniform(0.0, 2.0, n).astype(np.float32) if with_beta else np.zeros(0, np.float32)
    out["B"] = rng.uniform(0.1, 3.0, nv).astype(np.float32)
    out["A"] = rng.uniform(-1.0, 5.0, nv).astype(np.float32)
    out["M"] = rng.uniform(0.05, 50.0, nv).astype(np.float32)
    ns = rng.poisson(3.0, nv).astype(np.int16)
    ns[rng.random(nv) < 0.1] = -1
    out["NS"] = ns
    return out


def groups_of(z):
    return [dict(R=z[f"g{g}_R"], P=z[f"g{g}_P"], iz0=z[f"g{g}_iz0"], iy0=z[f"g{g}_iy0"], ix0=z[f"g{g}_ix0"],
                 rows=z[f"g{g}_rows"]) for g in range(int(z["n_groups"]))]


if __name__ == "__main__":
    import torch
    sys.path.insert(0, str(HERE))
    from refpath import import_reference
    import_reference()
    from xpg.forward import model as RM
    save = {}
    for k in range(len(CASES)):
        z = case_inputs(k)
        f0, f1, y0, ny, x0, nx = (int(v) for v in z["win"])
        n = int(z["n"])
        wm = RM.WindowModel.__new__(RM.WindowModel)
        wm.dev = torch.device("cpu")
        wm.win = RM.Window(f0=f0, f1=f1, nx=nx, ny=ny, rows=np.arange(n), groups=[], voxel_ids=[], x0=x0, y0=y0)
        wm.refl = {"x": np.zeros(n)}
        wm.width = dict(sd=0.01, sm=0.01, halo=None)
        wm.geom = np.zeros(8)
        wm.beta = None
        wm.cache = True
        wm.compact = False
        wm.items = []
        for g in groups_of(z):
            T_, m, Dz = g["R"].shape
            b = g["P"].shape[-1]
            terms = [(torch.from_numpy(g["R"][t]), torch.from_numpy(g["P"][t])) for t in range(T_)]
            wm.items.append(dict(rows=g["rows"], Dz=Dz, b=b, iz0=torch.from_numpy(g["iz0"]),
                                 iy0=torch.from_numpy(g["iy0"]), ix0=torch.from_numpy(g["ix0"]),
                                 _key=wm._key(), _terms=terms))
        I = torch.from_numpy(z["I"])
        beta = torch.from_numpy(z["beta"]) if z["beta"].size else None
        B = torch.from_numpy(z["B"])
        mu = wm.mu(I, B, beta=beta)
        M, A = torch.from_numpy(z["M"]), torch.from_numpy(z["A"])
        NS = torch.from_numpy(z["NS"])
        gr = wm.grad_ratio(A, M, NS)
        gn, fd = wm.grad_newton(M, NS)
        for key, v in z.items():
            save[f"c{k}_{key}"] = v
        save[f"c{k}_xpg_mu"] = mu.numpy()
        save[f"c{k}_xpg_grad_ratio"] = gr.numpy()
        save[f"c{k}_xpg_grad_newton"] = gn.numpy()
        save[f"c{k}_xpg_fisher_diag"] = fd.numpy()
    save["n_cases"] = np.int64(len(CASES))
    np.savez_compressed(HERE / "forward.npz", **save)
    print((HERE / "forward.npz").stat().st_size)
