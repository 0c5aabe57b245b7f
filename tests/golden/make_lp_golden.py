"""Makes lp_output.npz: XPG's own Lorentz-polarisation / absorption factors (`Geometry.lp_factor`,
`Geometry.absorption_factors`, `xpg/geometry.py:372-407`) and its INTEGRATE.HKL writer (`write_integrate_hkl`,
`xpg/io/legacy.py:140-182`) applied to the reference's integration results stored in the golden fixtures, with the
INTEGRATE stage's correction and row selection around them (`xpg/stage_integrate.py:408-431`, restated here because
the stage module imports gemmi, absent in this container; without gemmi XPG writes space group number 1).

Per case: the LP / absorption factor rlp of the kept lattice-0 rows, their indices, the row counts of the other lattices, and
the INTEGRATE.HKL header (without its DATE and Generated-by lines), the sha256 of its data records and the first
three records.

    python tests/golden/make_lp_golden.py        (needs the reference checkout importable)
"""
from __future__ import annotations

import hashlib
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

import golden_io as G  # noqa: E402

CASES = ("config1", "adaptive", "superpix", "binned", "crowded", "precision")


def _rows(refl, m):
    return {k: (v[m] if isinstance(v, np.ndarray) and v.shape[:1] == m.shape else v) for k, v in refl.items()}


def split_hkl(text):
    lines = text.splitlines()
    k = lines.index("!END_OF_HEADER")
    head = [ln for ln in lines[:k + 1] if not ln.startswith(("!OUTPUT_FILE=", "!Generated by"))]
    recs = lines[k + 1:]
    return head, recs


def main():
    from refpath import import_reference
    import_reference()
    from xpg.geometry import Geometry as RGeometry
    from xpg.io.legacy import write_integrate_hkl
    from xpg.models import Crystal as RCrystal, Experiment as RExperiment
    import make_golden as MG
    out = {}
    for case in CASES:
        z = G.load(case)
        refl = {k[4:]: z[k] for k in z if k.startswith("out_")}
        spec = G.spec_of(case)
        exp = MG._ref_experiment(spec, RGeometry, RCrystal, RExperiment)
        g = exp.geom
        zeta_l, pol = g.lp_factor(refl["S"])
        rlp = np.abs(zeta_l) / pol / g.absorption_factors(refl["S"])
        r = dict(refl)
        r["rlp"] = rlp
        r["I"] = r["iprf"] * rlp
        r["sig"] = np.sqrt(np.maximum(r["vprf"], 0)) * rlp
        r["Isum"] = r["isum"] * rlp
        r["sigsum"] = np.sqrt(np.maximum(r["vsum"], 0)) * rlp
        r["peak"] = 100 * np.clip(r["p_valid"] / np.maximum(r["p_total"], 1e-9), 0, 1) * r.get("coverage", 1.0)
        r["corr"] = 100 * np.nan_to_num(r["corr"])
        good = np.isfinite(r["I"]) & np.isfinite(r["sig"]) & (r["sig"] > 0)
        idx = np.flatnonzero(good)
        r = _rows(r, good)
        lat = r.get("lattice", np.zeros(len(r["I"]), int))
        main = _rows(r, lat == 0)
        for k in ("rlp",):                   # the rest follows from rlp and the inputs (the records pin it)
            out[f"{case}_{k}"] = main[k]
        out[f"{case}_keep"] = idx[lat == 0]
        out[f"{case}_n_extra"] = np.array([int((lat == k).sum()) for k in range(1, int(lat.max()) + 1 if lat.size
                                                                                 else 1)], np.int64)
        with tempfile.TemporaryDirectory() as d:
            p = Path(d) / "INTEGRATE.HKL"
            write_integrate_hkl(p, exp, main, (1, spec.nframes), spec.sigma_m, spec.sigma_d, "frame_?????.cbf")
            head, recs = split_hkl(p.read_text())
        out[f"{case}_hkl_head"] = np.array("\n".join(head))
        out[f"{case}_hkl_sha"] = np.array(hashlib.sha256("\n".join(recs).encode()).hexdigest())
        out[f"{case}_hkl_first"] = np.array("\n".join(recs[:3]))
        print(case, len(main["I"]), out[f"{case}_n_extra"])
    np.savez_compressed(HERE / "lp_output.npz", **out)


if __name__ == "__main__":
    main()
