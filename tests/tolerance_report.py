"""How many rows of each golden fixture the conditioning rules of tests/tolerance.py exempt or judge on their scale
floor, from the reference's own results in the fixture:

* m_d / m_m compared only where I/sigma >= 3 (`tolerance.meaningful`);
* pass-2 outputs compared only where >= 1% of the profile lies on valid pixels (`tolerance.meaningful`);
* summation and profile-fitted intensities judged against sigma instead of |I| where |I| < sigma (`tolerance.scale`).

    python tests/tolerance_report.py        (markdown table on stdout; CPU only)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

import golden_io as G  # noqa: E402


def counts(case):
    z = G.load(case)
    out = {k[4:]: np.asarray(v) for k, v in z.items() if k.startswith("out_")}
    n = out["x"].size
    isum, vsum = out["isum"].astype(float), out["vsum"].astype(float)
    iprf, vprf = out["iprf"].astype(float), out["vprf"].astype(float)
    fin = np.isfinite(iprf)
    weak_moments = ~(isum >= 3.0 * np.sqrt(np.maximum(vsum, 1e-6)))
    no_fit = fin & ~(out["p_valid"] >= 0.01 * out["p_total"])
    floor_sum = np.abs(isum) < np.sqrt(np.maximum(np.abs(vsum), 1.0))
    floor_prf = fin & (np.abs(iprf) < np.sqrt(np.maximum(np.abs(vprf), 1.0)))
    return dict(rows=n, moments_exempt=int(weak_moments.sum()), pass2_exempt=int(no_fit.sum()),
                isum_on_sigma=int(floor_sum.sum()), iprf_on_sigma=int(floor_prf.sum()))


def table():
    lines = ["| fixture | rows | m_d, m_m not compared (I/sigma < 3) | pass-2 outputs not compared (valid profile < 1%) "
             "| I_sum judged on sigma (abs(I) < sigma) | I_prf judged on sigma |", "|---|---|---|---|---|---|"]
    for case in G.CASES:
        c = counts(case)
        lines.append(f"| {case} | {c['rows']} | {c['moments_exempt']} | {c['pass2_exempt']} | {c['isum_on_sigma']} "
                     f"| {c['iprf_on_sigma']} |")
    return "\n".join(lines)


if __name__ == "__main__":
    print(table())
