"""Parity tolerances of the integration outputs.

The primary outputs (background, summation intensity and variance, profile-fitted intensity and variance) must
agree within 1e-5 relative of the reference, with an absolute floor of 1e-5 of the quantity's natural scale
where it can cancel to zero (an intensity near zero is judged against its sigma). Other floating outputs (moments,
correlations, fractions) carry the reference's own float32 summation error and are held to 1e-4 of their scale.
Integer outputs and masks are exact.
"""
from __future__ import annotations

import numpy as np

REL = 1e-5
REL_AUX = 1e-4


def scale(key, ref, row_ctx):
    """Absolute floor of a quantity (see module docstring); row_ctx holds the row's reference outputs."""
    ref = np.abs(np.asarray(ref, np.float64))
    if key in ("isum",):
        return np.sqrt(np.maximum(np.abs(row_ctx["vsum"]), 1.0))
    if key in ("iprf", "ipartner"):
        return np.sqrt(np.maximum(np.abs(row_ctx["vprf"]), 1.0))
    if key in ("corr", "rho", "p_fg", "frac_rec"):
        return 1.0
    if key == "p_valid":
        return np.abs(row_ctx["p_total"])
    if key in ("fz", "img2"):
        return np.sqrt(np.maximum(np.abs(row_ctx["vsum"]), 1.0))
    if key in ("m_d",):
        return np.float64(row_ctx["seff"]) ** 2
    if key in ("m_m",):
        return np.maximum(np.abs(np.float64(row_ctx["m_m"])), 1e-12) + np.float64(row_ctx["seff"]) ** 2
    if key in ("u1", "u2"):
        return np.max(np.abs(np.asarray(row_ctx[key])))
    if key == "J":
        return np.max(np.abs(np.asarray(row_ctx["J"])))
    if key in ("xo", "yo", "zo"):
        return 1.0
    return ref * 0.0


MAIN = {"bg", "nbg", "isum", "vsum", "vsum0", "iprf", "vprf", "vprf0"}


def meaningful(key, row_ctx):
    """The second moments of a spot are ratios of sums that cancel for reflections that are not significant:
    m_d / m_m are compared only where I/sigma >= 3 (XPG uses them only for strong spots, I/sigma > 10)."""
    if key in ("m_d", "m_m") and "isum" in row_ctx and "vsum" in row_ctx:
        return float(row_ctx["isum"]) >= 3.0 * np.sqrt(max(float(row_ctx["vsum"]), 1e-6))
    # profile-fit results of a reflection with under 1% of its profile on valid pixels are extrapolations from a
    # handful of pixels (XPG's PEAK is then < 1% and the reflection is rejected downstream)
    if key in PASS2 and "p_valid" in row_ctx and "p_total" in row_ctx:
        return float(row_ctx["p_valid"]) >= 0.01 * float(row_ctx["p_total"])
    return True


PASS2 = {"iprf", "vprf", "vprf0", "corr", "rho", "ipartner"}


def within(key, mine, ref, row_ctx, rel=None):
    """(ok, worst relative-to-scale error) of mine against ref."""
    if not meaningful(key, row_ctx):
        return True, 0.0
    mine = np.asarray(mine, np.float64)
    ref = np.asarray(ref, np.float64)
    r = rel if rel is not None else (REL if key in MAIN else REL_AUX)
    fl = scale(key, ref, row_ctx)
    tol = r * np.maximum(np.abs(ref), fl)
    err = np.abs(mine - ref)
    bad = ~((err <= tol) | (np.isnan(mine) & np.isnan(ref)))
    worst = float(np.max(err / np.maximum(np.maximum(np.abs(ref), fl), 1e-300))) if err.size else 0.0
    return (not bad.any()), worst
