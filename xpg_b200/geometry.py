"""Rotation-method diffraction geometry needed by the integration path (host side, float64 numpy).

Conventions are those of XPG (`xpg/geometry.py:1-17`): detector point (x, y) is continuous with the centre of
array element ix at x = ix + 1 (`PIX0`), the lab position of a detector point is an affine map per panel, the
spindle angle of the continuous frame coordinate z is phi(z) = phi0 + osc * (z - (starting_frame - 1)), and the
reciprocal basis A* has a*, b*, c* as its columns at phi = 0.

`Geometry` keeps the reference's attribute names (`xpg/geometry.py:123-150`) so that an XPG `Experiment` can be
handed to `xpg_b200.integrate` unchanged: the integration path reads only the attributes and methods defined here.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field, replace

import numpy as np

PIX0 = 1.0      # continuous coordinate of the centre of array element 0

_POOL = None


def _pool():
    global _POOL
    if _POOL is None:
        _POOL = ThreadPoolExecutor(max(1, min(16, len(os.sched_getaffinity(0)))))
    return _POOL


def row_chunks(n, min_rows=65536):
    """Contiguous row ranges for the host thread pool (numpy releases the GIL in its array loops)."""
    k = max(1, min(_pool()._max_workers, n // min_rows))
    e = np.linspace(0, n, k + 1).astype(int)
    return [(int(a), int(b)) for a, b in zip(e[:-1], e[1:])]


def par_rows(fn, n, min_rows=65536):
    """fn(a, b) over row ranges of [0, n) on the host thread pool, results in order. Element-wise work split this
    way is bit-identical to one call over all rows."""
    ch = row_chunks(n, min_rows)
    if len(ch) == 1:
        return [fn(0, n)]
    return list(_pool().map(lambda ab: fn(*ab), ch))


def unit(v):
    v = np.asarray(v, dtype=float)
    return v / np.linalg.norm(v)


def axis_angle_matrices(axis, angles):
    """Right-handed rotations about the unit vector `axis` by `angles` (radians), shape angles.shape + (3, 3)
    (Rodrigues' formula)."""
    k = unit(axis)
    ang = np.asarray(angles, float)
    K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    c = np.cos(ang)[..., None, None]
    s = np.sin(ang)[..., None, None]
    return c * np.eye(3) + s * K + (1.0 - c) * np.outer(k, k)


def cell_to_B(cell):
    """Reciprocal basis (columns a*, b*, c*) of a unit cell in the Busing-Levy frame: a along x, b in the xy plane."""
    a, b, c, al, be, ga = cell
    cal, cbe, cga = np.cos(np.radians([al, be, ga]))
    sga = np.sin(np.radians(ga))
    cx = c * cbe
    cy = c * (cal - cbe * cga) / sga
    cz = np.sqrt(max(c * c - cx * cx - cy * cy, 1e-12))
    real_rows = np.array([[a, 0.0, 0.0], [b * cga, b * sga, 0.0], [cx, cy, cz]])
    return np.linalg.inv(real_rows)


def random_orientation(rng):
    """Uniformly distributed rotation matrix from a random unit quaternion."""
    q = rng.normal(size=4)
    w, x, y, z = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


@dataclass
class Panel:
    """One detector segment (the legacy SEGMENT= record, `xpg/detector.py:36-60`): inclusive 1-based pixel
    rectangle, segment origin (pixels) and distance (mm) and its in-plane axes in the detector system."""
    x1: int
    x2: int
    y1: int
    y2: int
    orgx: float = 0.0
    orgy: float = 0.0
    distance: float = 0.0
    ex: np.ndarray = field(default_factory=lambda: np.array([1.0, 0.0, 0.0]))
    ey: np.ndarray = field(default_factory=lambda: np.array([0.0, 1.0, 0.0]))

    def frame(self, qx, qy):
        """(offset c, ex, ey) in the detector system; ey is made orthogonal to ex."""
        ex = unit(self.ex)
        ey = np.asarray(self.ey, float)
        ey = unit(ey - np.dot(ey, ex) * ex)
        ez = np.cross(ex, ey)
        return -qx * self.orgx * ex - qy * self.orgy * ey + self.distance * ez, ex, ey


def panel_maps(panels, orgx, orgy, distance, ed1, ed2, qx, qy):
    """Lab affine map of every panel: X(x, y) = P0 + (x - orgx) Bx + (y - orgy) By, each (K, 3).

    The arithmetic follows `xpg/detector.py:79-90` step for step, so that the float32 copies handed to the kernels
    are the reference's to the last bit."""
    fr = [p.frame(qx, qy) for p in panels]
    C = np.array([f[0] for f in fr])
    EX = np.array([f[1] for f in fr])
    EY = np.array([f[2] for f in fr])
    ed3 = np.cross(ed1, ed2)
    E = np.stack([ed1, ed2, ed3], axis=0)
    Bx = qx * (EX @ E)
    By = qy * (EY @ E)
    origin = np.stack([-qx * orgx * np.ones(()), -qy * orgy * np.ones(()), distance * np.ones(())])
    A = (C + origin) @ E
    return A + orgx * Bx + orgy * By, Bx, By


def parallax_shift(e, u1, u2, un, t, mu):
    """Mean absorption depth of a ray e in a sensor of thickness t (attenuation mu), projected on the panel axes."""
    cosa = np.clip(np.sum(e * un, -1), 1e-3, 1.0)
    L = t / cosa
    muL = mu * L
    lbar = 1.0 / mu - L * np.exp(-muL) / np.maximum(-np.expm1(-muL), 1e-12)
    return lbar * np.sum(e * u1, -1), lbar * np.sum(e * u2, -1)


def _bilinear_table(tab, x, y):
    ny, nx = tab.shape
    fx = np.clip(x - 1.0, 0, nx - 1.000001)
    fy = np.clip(y - 1.0, 0, ny - 1.000001)
    ix = np.floor(fx).astype(np.int32)
    iy = np.floor(fy).astype(np.int32)
    ix1 = np.minimum(ix + 1, nx - 1)
    iy1 = np.minimum(iy + 1, ny - 1)
    tx, ty = fx - ix, fy - iy
    return (tab[iy, ix] * (1 - tx) * (1 - ty) + tab[iy, ix1] * tx * (1 - ty)
            + tab[iy1, ix] * (1 - tx) * ty + tab[iy1, ix1] * tx * ty)


@dataclass
class Geometry:
    wavelength: float
    beam: np.ndarray
    axis: np.ndarray
    orgx: float
    orgy: float
    distance: float
    ed1: np.ndarray
    ed2: np.ndarray
    qx: float
    qy: float
    nx: int
    ny: int
    phi0: float
    osc: float
    starting_frame: int = 1
    polarization_fraction: float = 0.5
    polarization_normal: np.ndarray = field(default_factory=lambda: np.array([0.0, 1.0, 0.0]))
    sensor_thickness: float = 0.0
    mu: float = 0.0
    segments: list | None = None
    geo_corr: tuple | None = None

    def copy(self, **kw):
        return replace(self, **kw)

    @property
    def ed3(self):
        return np.cross(self.ed1, self.ed2)

    @property
    def s0(self):
        return self.beam / self.wavelength

    @property
    def has_parallax(self):
        return self.sensor_thickness > 0 and self.mu > 0

    @property
    def segmented(self):
        return bool(self.segments)

    def z_to_phi(self, z):
        return self.phi0 + self.osc * (np.asarray(z) - (self.starting_frame - 1))

    def phi_to_z(self, phi):
        return (np.asarray(phi) - self.phi0) / self.osc + (self.starting_frame - 1)

    def panel_list(self):
        return self.segments if self.segments else [Panel(1, max(self.nx, 1), 1, max(self.ny, 1))]

    def panels(self):
        return panel_maps(self.panel_list(), self.orgx, self.orgy, self.distance, unit(self.ed1), unit(self.ed2),
                          self.qx, self.qy)

    def segmap(self):
        """(ny, nx) int16 panel index of every pixel, -1 in gaps; None for a single panel."""
        if not self.segmented:
            return None
        m = np.full((self.ny, self.nx), -1, np.int16)
        for k, s in enumerate(self.segments):
            m[max(s.y1 - 1, 0):min(s.y2, self.ny), max(s.x1 - 1, 0):min(s.x2, self.nx)] = k
        return m

    def _segment_of(self, x, y):
        if not self.segmented:
            return np.zeros(np.shape(x), int)
        m = self.segmap()
        ix = np.clip(np.floor(np.asarray(x, float) - 0.5).astype(np.int32), 0, m.shape[1] - 1)
        iy = np.clip(np.floor(np.asarray(y, float) - 0.5).astype(np.int32), 0, m.shape[0] - 1)
        return m[iy, ix].astype(int)

    def _corrected(self, x, y):
        if self.geo_corr is None:
            return x, y
        return x + _bilinear_table(self.geo_corr[0], x, y), y + _bilinear_table(self.geo_corr[1], x, y)

    def pixel_to_lab(self, x, y):
        """Lab position (mm) of the sensor entry point of the ray recorded at detector point (x, y)."""
        x = np.asarray(x, float)
        y = np.asarray(y, float)
        if not self.segmented and self.geo_corr is None and not self.has_parallax:
            return (self.qx * (x[..., None] - self.orgx) * self.ed1 + self.qy * (y[..., None] - self.orgy) * self.ed2
                    + self.distance * self.ed3)
        P0, Bx, By = self.panels()
        k = np.maximum(self._segment_of(x, y), 0)
        xc, yc = self._corrected(x, y)
        P0k, Bxk, Byk = P0[k], Bx[k], By[k]
        lab = lambda a, b: P0k + (a - self.orgx)[..., None] * Bxk + (b - self.orgy)[..., None] * Byk
        X = lab(xc, yc)
        if self.has_parallax:
            u1, u2 = Bxk / self.qx, Byk / self.qy
            un = np.cross(u1, u2)
            for _ in range(4):
                e = X / np.linalg.norm(X, axis=-1, keepdims=True)
                d1, d2 = parallax_shift(e, u1, u2, un, self.sensor_thickness, self.mu)
                X = lab(xc - d1 / self.qx, yc - d2 / self.qy)
        return X

    def pixel_to_s(self, x, y):
        X = self.pixel_to_lab(x, y)
        return X / (np.linalg.norm(X, axis=-1, keepdims=True) * self.wavelength)

    def s_to_pixel(self, S):
        """Detector point (x, y) hit by the rays S (nan where a ray meets no panel)."""
        S = np.asarray(S, float)
        P0, Bx, By = self.panels()
        panels = self.panel_list()
        x = np.full(S.shape[:-1], np.nan)
        y = np.full(S.shape[:-1], np.nan)
        for k, pan in enumerate(panels):
            n = np.cross(Bx[k], By[k])
            with np.errstate(divide="ignore", invalid="ignore"):
                t = (P0[k] @ n) / (S @ n)
            P = t[..., None] * S - P0[k]
            xk = self.orgx + (P @ Bx[k]) / (Bx[k] @ Bx[k])
            yk = self.orgy + (P @ By[k]) / (By[k] @ By[k])
            hit = np.isfinite(t) & (t > 0)
            if self.has_parallax:
                u1, u2 = Bx[k] / self.qx, By[k] / self.qy
                e = S / np.linalg.norm(S, axis=-1, keepdims=True)
                with np.errstate(invalid="ignore"):
                    d1, d2 = parallax_shift(e, u1, u2, np.cross(u1, u2), self.sensor_thickness, self.mu)
                xk = xk + d1 / self.qx
                yk = yk + d2 / self.qy
            if self.geo_corr is not None:
                xr, yr = xk, yk
                for _ in range(4):           # fixed-point inversion of the distortion table
                    xr = xk - _bilinear_table(self.geo_corr[0], xr, yr)
                    yr = yk - _bilinear_table(self.geo_corr[1], xr, yr)
                xk, yk = xr, yr
            if self.segmented:
                hit &= (xk >= pan.x1 - 0.5) & (xk < pan.x2 + 0.5) & (yk >= pan.y1 - 0.5) & (yk < pan.y2 + 0.5)
            hit &= np.isnan(x)
            x = np.where(hit, xk, x)
            y = np.where(hit, yk, y)
        return x, y

    def lp_factor(self, S):
        """(Lorentz zeta, polarisation P) of diffracted rays S; corrected intensities are I * |zeta| / P."""
        e = S / np.linalg.norm(S, axis=-1, keepdims=True)
        e0 = self.beam
        zeta = np.cross(e, e0) @ self.axis
        n = self.polarization_normal - np.dot(self.polarization_normal, e0) * e0
        n = n / np.linalg.norm(n)
        emain = np.cross(n, e0)
        f = self.polarization_fraction
        return zeta, f * (1 - (e @ emain) ** 2) + (1 - f) * (1 - (e @ n) ** 2)

    def absorption_factors(self, S):
        """Sensor absorption efficiency of rays S (1 without a sensor model). Air absorption, which XPG's stage
        adds from its attenuation tables, is not modelled here."""
        e = S / np.linalg.norm(S, axis=-1, keepdims=True)
        f = np.ones(e.shape[:-1])
        if self.has_parallax:
            cosn = e @ self.ed3
            f = f * -np.expm1(-self.mu * self.sensor_thickness / np.clip(cosn, 1e-3, 1.0))
        return f


@dataclass
class Crystal:
    U: np.ndarray
    cell: np.ndarray
    space_group: str = "P 1"

    @property
    def Astar(self):
        return self.U @ cell_to_B(self.cell)


@dataclass
class Experiment:
    geom: Geometry
    crystal: Crystal


def generate_hkl(Astar, dmin, dmax=1e9):
    """Miller indices with dmin <= d < dmax, 000 excluded (`xpg/geometry.py:468-479`)."""
    real = np.linalg.inv(Astar)
    hmax = [int(np.ceil(np.linalg.norm(real[i]) / dmin)) for i in range(3)]
    axes = [np.arange(-m, m + 1) for m in hmax]

    def part(a, b):             # h values axes[0][a:b] (the grid is h-major: chunks keep the order)
        H = np.stack(np.meshgrid(axes[0][a:b], axes[1], axes[2], indexing="ij"), -1).reshape(-1, 3)
        p = H @ Astar.T
        q2 = np.einsum("ij,ij->i", p, p)
        return H[(q2 <= 1.0 / dmin ** 2) & (q2 > 1.0 / dmax ** 2)].astype(np.int32)
    return np.concatenate(par_rows(part, len(axes[0]), min_rows=8))


def diffraction_angles(geom, p0):
    """Both spindle angles (radians) at which each p0 meets the Ewald sphere, and whether it does.

    R(phi) p0 = p_par + cos(phi) p_perp + sin(phi) (m x p0); the Laue condition |s0 + p|^2 = |s0|^2 becomes
    a cos(phi) + b sin(phi) = c with a = s0.p_perp, b = s0.(m x p0), c = -|p0|^2 / 2 - s0.p_par."""
    m = geom.axis
    s0 = geom.s0
    p0 = np.asarray(p0, float)
    p_par = (p0 @ m)[:, None] * m
    a = (p0 - p_par) @ s0
    b = np.cross(m, p0) @ s0
    c = -0.5 * np.einsum("ij,ij->i", p0, p0) - p_par @ s0
    r = np.hypot(a, b)
    with np.errstate(invalid="ignore", divide="ignore"):
        q = c / r
    ok = np.abs(q) <= 1.0
    base = np.arctan2(b, a)
    half = np.arccos(np.clip(q, -1, 1))
    return base + half, base - half, ok


def predict_reflections(geom, Astar, dmin, dmax=1e9, z_range=None, hkl=None):
    """Predicted reflections of a rotation sweep: dict of hkl, x, y, z (frame coordinate), phi (deg), S (lab, at
    diffraction), zeta (Lorentz) and polarization, for z in z_range (`xpg/geometry.py:505-545`)."""
    if hkl is None:
        hkl = generate_hkl(Astar, dmin, dmax)
    p0 = hkl @ Astar.T
    ang = par_rows(lambda a, b: diffraction_angles(geom, p0[a:b]), len(p0))
    pa, pb, ok = (np.concatenate([x[i] for x in ang]) for i in range(3))
    if z_range is None:
        z_range = (geom.starting_frame - 1, geom.starting_frame - 1 + 360.0 / abs(geom.osc))
    lo, hi = sorted(geom.z_to_phi(np.array(z_range, float)))
    H_all, ph_all, S_all = [], [], []
    for sol in (pa, pb):
        ph = np.degrees(sol[ok])
        ph = lo + np.mod(ph - lo, 360.0)
        for turn in (0.0, 360.0):
            phs = ph + turn
            sel = (phs >= lo) & (phs < hi)
            if not sel.any():
                continue
            ph_sel, p_sel = phs[sel], p0[ok][sel]
            S_all.append(np.concatenate(par_rows(
                lambda a, b: np.einsum("nij,nj->ni", axis_angle_matrices(geom.axis, np.radians(ph_sel[a:b])),
                                       p_sel[a:b]) + geom.s0, len(ph_sel))))
            H_all.append(hkl[ok][sel])
            ph_all.append(phs[sel])
    if not H_all:
        e = np.zeros(0)
        return dict(hkl=np.zeros((0, 3), np.int32), phi=e, S=np.zeros((0, 3)), x=e, y=e, z=e, zeta=e, polarization=e)
    res = dict(hkl=np.concatenate(H_all), phi=np.concatenate(ph_all), S=np.concatenate(S_all))
    S = res["S"]
    xy = par_rows(lambda a, b: geom.s_to_pixel(S[a:b]), len(S))
    res["x"], res["y"] = np.concatenate([v[0] for v in xy]), np.concatenate([v[1] for v in xy])
    res["z"] = geom.phi_to_z(res["phi"])
    lp = par_rows(lambda a, b: geom.lp_factor(S[a:b]), len(S))
    res["zeta"], res["polarization"] = np.concatenate([v[0] for v in lp]), np.concatenate([v[1] for v in lp])
    keep = np.isfinite(res["x"])
    return {k: v[keep] for k, v in res.items()}


def centring_allowed(hkl, space_group):
    """Reflections allowed by the lattice centring of a Hermann-Mauguin symbol (first letter): P, C, A, B, I, F, R
    (obverse). XPG asks gemmi for the centring vectors (`xpg/integrate.py:86-98`); the rule is the same."""
    sym = str(space_group).strip().upper()[:1]
    h, k, l = (np.asarray(hkl)[:, i] for i in range(3))
    if sym == "C":
        return (h + k) % 2 == 0
    if sym == "A":
        return (k + l) % 2 == 0
    if sym == "B":
        return (h + l) % 2 == 0
    if sym == "I":
        return (h + k + l) % 2 == 0
    if sym == "F":
        return ((h + k) % 2 == 0) & ((k + l) % 2 == 0)
    if sym == "R":
        return (-h + k + l) % 3 == 0
    return np.ones(len(h), bool)
