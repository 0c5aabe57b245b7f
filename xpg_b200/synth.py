"""Seeded synthetic rotation sweeps: the detector, crystal and beam of a workload, its predicted reflections and
uint32 frames with Eiger-style encoding (module gaps and flagged pixels at 0xFFFFFFFF, counts >= the overload
threshold overloaded).

The spot model follows XPG's simulator (`xpg/simulate.py:251-385`): Wilson acentric intensities, Gaussian spots of
width sigma_D in the detector plane (stretched radially by the obliquity), a frame-integrated Gaussian rocking
curve of width sigma_M / |zeta|, a flat Poisson background with a radial ramp, and Poisson noise. Intensities are a
deterministic hash of the Miller index, so any frame range of a sweep renders the same crystal.

`render_frames` is the host (numpy) generator for CPU-sized sweeps; `xpg_b200.native.synth_frames` renders the
same model on the device for sweeps whose stack does not fit in host memory.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np
from scipy.special import erf

from .geometry import (PIX0, Crystal, Experiment, Geometry, cell_to_B, centring_allowed, predict_reflections,
                       random_orientation, unit)

GAP_VALUE = np.uint32(0xFFFFFFFF)


@dataclass
class SweepSpec:
    name: str = "small"
    nx: int = 256
    ny: int = 272
    qx: float = 0.172
    distance: float = 80.0
    wavelength: float = 1.0
    orgx: float | None = None       # beam centre (pixels); default: detector centre
    orgy: float | None = None
    osc: float = 0.2
    nframes: int = 30
    phi0: float = 0.0
    cell: tuple = (41.3, 52.7, 60.1, 90.0, 90.0, 90.0)
    space_group: str = "P 21 21 21"
    sigma_d: float = 0.03           # deg
    sigma_m: float = 0.1            # deg
    wilson_b: float = 20.0
    mean_i0: float = 50.0           # mean photons of a low-resolution reflection
    background: float = 0.5         # mean counts / pixel at the beam centre
    ramp: float = 0.5               # background grows by this fraction towards the detector corners
    dmin: float | None = None       # default: detector edge
    gaps: bool = True
    overload: int = 1 << 20
    hot_fraction: float = 0.0       # reflections scaled up so that their peaks overload
    weak_fraction: float = 0.0      # reflections with mean 2 photons
    dead_fraction: float = 0.0      # reflections covered by a dead (masked) rectangle over > 40% of their box
    seed: int = 1
    n_regions_xy: int = 3
    block_frames: int = 0           # phi block length in frames (0: one block)
    sensor_thickness: float = 0.0   # mm; > 0 with mu > 0 models sensor parallax
    mu: float = 0.0                 # sensor attenuation (1/mm)
    beam: tuple = (0.0, 0.0, 1.0)
    axis: tuple = (1.0, 0.0, 0.0)
    U: np.ndarray | None = field(default=None, repr=False)

    def geometry(self) -> Geometry:
        return Geometry(wavelength=self.wavelength, beam=unit(self.beam), axis=unit(self.axis),
                        orgx=self.nx / 2.0 if self.orgx is None else self.orgx,
                        orgy=self.ny / 2.0 if self.orgy is None else self.orgy,
                        distance=self.distance, ed1=np.array([1.0, 0.0, 0.0]), ed2=np.array([0.0, 1.0, 0.0]),
                        qx=self.qx, qy=self.qx, nx=self.nx, ny=self.ny, phi0=self.phi0, osc=self.osc,
                        starting_frame=1, polarization_fraction=0.99, polarization_normal=np.array([0.0, 1.0, 0.0]),
                        sensor_thickness=self.sensor_thickness, mu=self.mu)

    def orientation(self):
        if self.U is not None:
            return np.asarray(self.U, float)
        return random_orientation(np.random.default_rng(self.seed))

    def experiment(self) -> Experiment:
        return Experiment(self.geometry(), Crystal(U=self.orientation(), cell=np.array(self.cell, float),
                                                   space_group=self.space_group))

    def resolution_limit(self):
        """dmin: the given value, else the resolution at the detector edge closest to the corners' worst."""
        if self.dmin:
            return float(self.dmin)
        g = self.geometry()
        cx = np.array([0.5, self.nx + 0.5, 0.5, self.nx + 0.5])
        cy = np.array([0.5, 0.5, self.ny + 0.5, self.ny + 0.5])
        S = g.pixel_to_s(cx, cy)
        return float((1.0 / np.linalg.norm(S - g.s0, axis=-1)).min())

    def block_edges(self):
        """Phi block edges in continuous frame coordinates (block b covers z in [edges[b], edges[b+1]))."""
        n = self.nframes
        if not self.block_frames or self.block_frames >= n:
            return np.array([0.0, float(n)])
        e = list(range(0, n, self.block_frames)) + [n]
        return np.array(e, float)

    def gap_mask(self):
        """(ny, nx) bool, True where the detector has a module gap (Pilatus / Eiger module pitch)."""
        m = np.zeros((self.ny, self.nx), bool)
        if self.gaps:
            for y0 in range(195, self.ny, 212):
                m[y0:y0 + 17, :] = True
            for x0 in range(487, self.nx, 494):
                m[:, x0:x0 + 7] = True
        return m


def config1(**kw) -> SweepSpec:
    """Plain small sweep: 1030 x 1065 px of 75 um at 150 mm, lambda 1.0 A, 100 x 0.1 deg, P 43 21 2 79/79/38 A,
    sigma_M 0.1 deg, sigma_D 0.03 deg, Wilson B 20 with mean 50 photons, background 0.5 + radial ramp, 3 x 3
    regions, one phi block."""
    base = dict(name="config1", nx=1030, ny=1065, qx=0.075, distance=150.0, wavelength=1.0, osc=0.1, nframes=100,
                cell=(79.0, 79.0, 38.0, 90.0, 90.0, 90.0), space_group="P 43 21 2", sigma_d=0.03, sigma_m=0.1,
                wilson_b=20.0, mean_i0=50.0, background=0.5, ramp=0.5, seed=1, n_regions_xy=3)
    base.update(kw)
    return SweepSpec(**base)


def config2(**kw) -> SweepSpec:
    """Plain sweep at scale: 4148 x 4362 px (16M) of 75 um at 120 mm, lambda 0.98 A, 3600 x 0.1 deg, P 21 21 21
    60/85/120 A, sigma_M 0.15 deg, sigma_D 0.03 deg, Wilson B 25, background 0.2, 5 x 5 regions, phi blocks of 360
    frames."""
    base = dict(name="config2", nx=4148, ny=4362, qx=0.075, distance=120.0, wavelength=0.98, osc=0.1, nframes=3600,
                cell=(60.0, 85.0, 120.0, 90.0, 90.0, 90.0), space_group="P 21 21 21", sigma_d=0.03, sigma_m=0.15,
                wilson_b=25.0, mean_i0=50.0, background=0.2, ramp=0.5, seed=2, n_regions_xy=5, block_frames=360)
    base.update(kw)
    return SweepSpec(**base)


def config3(**kw) -> SweepSpec:
    """Precision form on config 1's sweep: 5% weak reflections (mean 2 photons), 2% shoeboxes > 40% masked."""
    return config1(name="config3", weak_fraction=0.05, dead_fraction=0.02, seed=3, **kw)


CONFIG4_DETECTORS = ((1030, 1065), (2068, 2162), (4148, 4362))
CONFIG4_CELLS = (((60.0, 85.0, 120.0, 90.0, 90.0, 90.0), "P 21 21 21"),
                 ((150.0, 60.0, 90.0, 90.0, 105.0, 90.0), "C 1 2 1"),
                 ((100.0, 100.0, 200.0, 90.0, 90.0, 120.0), "P 65 2 2"))


def config4(seed=4, n_sweeps=12, **kw):
    """Batched workload: n_sweeps sweeps with frames drawn log-uniform in 50..3600, a detector from
    CONFIG4_DETECTORS (75 um pixels at 120 mm, lambda 0.98 A), a cell from CONFIG4_CELLS, sigma_M uniform in
    0.05..0.5 deg; phi blocks of 360 frames, background 0.2, Wilson B 25. Seeded: the same list every call."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_sweeps):
        nf = int(round(np.exp(rng.uniform(np.log(50.0), np.log(3600.0)))))
        nx, ny = CONFIG4_DETECTORS[int(rng.integers(len(CONFIG4_DETECTORS)))]
        cell, sg = CONFIG4_CELLS[int(rng.integers(len(CONFIG4_CELLS)))]
        sm = float(rng.uniform(0.05, 0.5))
        base = dict(name=f"config4-{k}", nx=nx, ny=ny, qx=0.075, distance=120.0, wavelength=0.98, osc=0.1,
                    nframes=nf, cell=cell, space_group=sg, sigma_d=0.03, sigma_m=sm, wilson_b=25.0, mean_i0=50.0,
                    background=0.2, ramp=0.5, seed=100 + 17 * seed + k, n_regions_xy=5 if nx > 2000 else 3,
                    block_frames=360)
        base.update(kw)
        out.append(SweepSpec(**base))
    return out


def config5(seed=5, n_sweeps=4, nframes=3600, **kw):
    """Served workload: n_sweeps concurrent sweeps of config 2's geometry (4148 x 4362 px, 75 um at 120 mm, lambda
    0.98 A, 0.1 deg frames, sigma_M 0.15 deg, background 0.2), cells from CONFIG4_CELLS, 50-frame wedges."""
    out = []
    for k in range(n_sweeps):
        cell, sg = CONFIG4_CELLS[k % len(CONFIG4_CELLS)]
        base = dict(name=f"config5-{k}", nx=4148, ny=4362, qx=0.075, distance=120.0, wavelength=0.98, osc=0.1,
                    nframes=nframes, cell=cell, space_group=sg, sigma_d=0.03, sigma_m=0.15, wilson_b=25.0,
                    mean_i0=50.0, background=0.2, ramp=0.5, seed=200 + 17 * seed + k, n_regions_xy=5,
                    block_frames=360)
        base.update(kw)
        out.append(SweepSpec(**base))
    return out


def _hash_unit(keys, salt):
    """Deterministic uniforms in (0, 1) from int64 keys (splitmix64 finaliser)."""
    with np.errstate(over="ignore"):
        x = np.asarray(keys, np.uint64) * np.uint64(0x9E3779B97F4A7C15) + np.uint64((salt * 0x632BE59BD9B4E019) % 2 ** 64)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return ((x >> np.uint64(11)).astype(np.float64) + 0.5) / float(2 ** 53)


def reflection_table(spec: SweepSpec, z_margin=5.0, z_range=None):
    """Predicted reflections of the sweep (z in [-margin, nframes + margin), or in z_range) with their true photon
    counts and the spot widths used to render them."""
    exp = spec.experiment()
    g = exp.geom
    A = exp.crystal.Astar
    dmin = spec.resolution_limit()
    from .geometry import generate_hkl
    hkl = generate_hkl(A, dmin)
    hkl = hkl[centring_allowed(hkl, spec.space_group)]
    zr = (-z_margin, spec.nframes + z_margin) if z_range is None else z_range
    pr = predict_reflections(g, A, dmin, z_range=zr, hkl=hkl)
    key = ((pr["hkl"][:, 0].astype(np.int64) + 1024) << 22) + ((pr["hkl"][:, 1].astype(np.int64) + 1024) << 11) \
        + (pr["hkl"][:, 2].astype(np.int64) + 1024)
    d = 1.0 / np.linalg.norm(pr["S"] - g.s0, axis=1)
    mean = spec.mean_i0 * np.exp(-0.5 * spec.wilson_b / d ** 2)
    I = -np.log(_hash_unit(key, spec.seed * 7 + 1)) * mean
    u = _hash_unit(key, spec.seed * 7 + 2)
    I = np.where(u < spec.weak_fraction, -np.log(_hash_unit(key, spec.seed * 7 + 3)) * 2.0, I)
    hot = (u >= spec.weak_fraction) & (u < spec.weak_fraction + spec.hot_fraction)
    I = np.where(hot, 2.0e7, I)
    e1 = np.cross(pr["S"], g.s0)
    e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
    zeta_u = np.abs(e1 @ g.axis)
    zl = np.abs(pr["zeta"])
    keep = (zl > 1e-3) & (zeta_u > 0.03)
    pr = {k: v[keep] for k, v in pr.items()}
    I, key, zeta_u, zl = I[keep], key[keep], zeta_u[keep], zl[keep]
    counts = I * pr["polarization"] / zl
    X = g.pixel_to_lab(pr["x"], pr["y"])
    L = np.linalg.norm(X, axis=1)
    cosa = (X @ g.ed3) / L
    sig_t = L * np.radians(spec.sigma_d) / spec.qx
    pr.update(I_true=I, counts=counts, key=key, sig_t=sig_t, sig_r=sig_t / cosa,
              sig_z=spec.sigma_m / zeta_u / spec.osc)
    return exp, pr


def background_image(spec: SweepSpec):
    g = spec.geometry()
    ys, xs = np.mgrid[0:spec.ny, 0:spec.nx]
    r = np.hypot(xs + PIX0 - g.orgx, ys + PIX0 - g.orgy)
    return (spec.background * (1.0 + spec.ramp * r / max(r.max(), 1.0))).astype(np.float64)


def dead_rectangles(spec: SweepSpec, table):
    """Dead (masked) rectangles over `dead_fraction` of the reflections, covering about half of their box."""
    if spec.dead_fraction <= 0:
        return []
    u = _hash_unit(table["key"], spec.seed * 7 + 5)
    pick = np.flatnonzero(u < spec.dead_fraction)
    out = []
    for i in pick:
        h = int(np.ceil(5 * table["sig_r"][i])) + 2
        x0 = int(np.floor(table["x"][i] - 1.0))
        y0 = int(np.floor(table["y"][i] - 1.0))
        out.append((max(x0 - h, 0), min(x0 + 1, spec.nx), max(y0 - h, 0), min(y0 + h + 1, spec.ny)))
    return out


def expected_frame(spec: SweepSpec, table, f, bg=None):
    """Expected counts of frame f (1-based): background plus every spot recorded on it."""
    img = background_image(spec) if bg is None else bg.copy()
    z0, z1 = f - 1.0, float(f)
    zc, sz = table["z"], table["sig_z"]
    act = np.flatnonzero((zc + 5 * sz > z0) & (zc - 5 * sz < z1))
    if act.size == 0:
        return img
    fz = 0.5 * (erf((z1 - zc[act]) / (np.sqrt(2) * sz[act])) - erf((z0 - zc[act]) / (np.sqrt(2) * sz[act])))
    x, y = table["x"][act], table["y"][act]
    st, sr = table["sig_t"][act], table["sig_r"][act]
    g = spec.geometry()
    rdir = np.c_[x - g.orgx, y - g.orgy]
    rn = np.linalg.norm(rdir, axis=1, keepdims=True)
    rdir = np.where(rn > 1e-6, rdir / np.maximum(rn, 1e-6), np.array([[1.0, 0.0]]))
    half = int(np.clip(np.ceil(4.5 * sr.max()), 4, 60))
    offs = np.arange(-half, half + 1)
    ix = np.floor(x - PIX0 + 0.5).astype(int)
    iy = np.floor(y - PIX0 + 0.5).astype(int)
    px = ix[:, None] + offs[None]
    py = iy[:, None] + offs[None]
    sub = (np.arange(2) + 0.5) / 2 - 0.5
    dens = 0.0
    for sy in sub:
        for sx in sub:
            dx = (px + PIX0 + sx - x[:, None])[:, None, :]
            dy = (py + PIX0 + sy - y[:, None])[:, :, None]
            ur = dx * rdir[:, 0, None, None] + dy * rdir[:, 1, None, None]
            ut = -dx * rdir[:, 1, None, None] + dy * rdir[:, 0, None, None]
            dens = dens + np.exp(-0.5 * ((ur / sr[:, None, None]) ** 2 + (ut / st[:, None, None]) ** 2))
    dens = dens / 4.0 / (2 * np.pi * sr * st)[:, None, None]
    val = (table["counts"][act] * fz)[:, None, None] * dens
    PY = np.broadcast_to(py[:, :, None], val.shape)
    PX = np.broadcast_to(px[:, None, :], val.shape)
    ok = (PX >= 0) & (PX < spec.nx) & (PY >= 0) & (PY < spec.ny)
    np.add.at(img, (PY[ok], PX[ok]), val[ok])
    return img


def render_frames(spec: SweepSpec, frames=None, table=None):
    """uint32 frames (len(frames), ny, nx) of the sweep (frames 1-based; default all). Gaps and dead rectangles are
    0xFFFFFFFF; Poisson counts are drawn from a generator seeded by (seed, frame), so any subset of frames is
    reproducible on its own."""
    if table is None:
        _, table = reflection_table(spec)
    frames = list(range(1, spec.nframes + 1)) if frames is None else list(frames)
    bg = background_image(spec)
    gaps = spec.gap_mask()
    for (x0, x1, y0, y1) in dead_rectangles(spec, table):
        gaps[y0:y1, x0:x1] = True
    out = np.empty((len(frames), spec.ny, spec.nx), np.uint32)
    for i, f in enumerate(frames):
        lam = expected_frame(spec, table, f, bg)
        rng = np.random.default_rng([spec.seed, int(f)])
        c = rng.poisson(lam)
        c = np.minimum(c, 0xFFFFFFFE).astype(np.uint32)
        c[gaps] = GAP_VALUE
        out[i] = c
    return out


def render_window(spec: SweepSpec, table, frames, y0, y1, x0, x1):
    """uint32 counts (len(frames), y1 - y0, x1 - x0) of a detector window [y0, y1) x [x0, x1) (array indices) over the
    given frames (1-based): the same model as `render_frames` (background with its ramp, the spots reaching the
    window, Poisson noise seeded by (seed, frame, window origin), module gaps flagged) without rendering whole
    frames. Dead rectangles are not applied."""
    g = spec.geometry()
    ys, xs = np.mgrid[y0:y1, x0:x1]
    cx = np.array([1.0, spec.nx, 1.0, spec.nx])
    cy = np.array([1.0, 1.0, spec.ny, spec.ny])
    rmax = max(np.hypot(cx - g.orgx, cy - g.orgy).max(), 1.0)
    bg = spec.background * (1.0 + spec.ramp * np.hypot(xs + PIX0 - g.orgx, ys + PIX0 - g.orgy) / rmax)
    near = np.flatnonzero((table["x"] > x0 - 62) & (table["x"] < x1 + 62) & (table["y"] > y0 - 62) &
                          (table["y"] < y1 + 62))
    sub = {k: np.asarray(v)[near] for k, v in table.items() if np.ndim(v) >= 1 and len(v) == len(table["x"])}
    gaps = spec.gap_mask()[y0:y1, x0:x1] if spec.gaps else np.zeros((y1 - y0, x1 - x0), bool)
    out = np.empty((len(frames), y1 - y0, x1 - x0), np.uint32)
    sub_off = (np.arange(2) + 0.5) / 2 - 0.5
    for i, f in enumerate(frames):
        lam = bg.copy()
        z0, z1 = f - 1.0, float(f)
        zc, sz = sub["z"], sub["sig_z"]
        for r in np.flatnonzero((zc + 5 * sz > z0) & (zc - 5 * sz < z1)):
            fz = 0.5 * (erf((z1 - zc[r]) / (np.sqrt(2) * sz[r])) - erf((z0 - zc[r]) / (np.sqrt(2) * sz[r])))
            x, y, st, sr = sub["x"][r], sub["y"][r], sub["sig_t"][r], sub["sig_r"][r]
            rd = np.array([x - g.orgx, y - g.orgy])
            rn = np.linalg.norm(rd)
            rd = rd / rn if rn > 1e-6 else np.array([1.0, 0.0])
            half = int(np.clip(np.ceil(4.5 * sr), 4, 60))
            ix, iy = int(np.floor(x - PIX0 + 0.5)), int(np.floor(y - PIX0 + 0.5))
            px = np.arange(max(ix - half, x0), min(ix + half + 1, x1))
            py = np.arange(max(iy - half, y0), min(iy + half + 1, y1))
            if not px.size or not py.size:
                continue
            dens = 0.0
            for oy in sub_off:
                for ox in sub_off:
                    dx = (px + PIX0 + ox - x)[None, :]
                    dy = (py + PIX0 + oy - y)[:, None]
                    ur, ut = dx * rd[0] + dy * rd[1], -dx * rd[1] + dy * rd[0]
                    dens = dens + np.exp(-0.5 * ((ur / sr) ** 2 + (ut / st) ** 2))
            lam[py[0] - y0:py[-1] + 1 - y0, px[0] - x0:px[-1] + 1 - x0] += \
                sub["counts"][r] * fz * dens / 4.0 / (2 * np.pi * sr * st)
        c = np.random.default_rng([spec.seed, int(f), int(y0), int(x0)]).poisson(lam)
        c = np.minimum(c, 0xFFFFFFFE).astype(np.uint32)
        c[gaps] = GAP_VALUE
        out[i] = c
    return out


def encode_frame(raw, overload, min_valid=0, mask=None):
    """The float32 frame XPG's image readers hand to integration (`xpg/io/images.py:72-102`, Eiger
    `:408-419`): counts as float32, overloaded (raw >= overload) -2, flagged (raw == 0xFFFFFFFF) or below
    min_valid -1 (masked wins over overloaded), then the integration mask ceiling (`xpg/integrate.py:667-680`):
    masked pixels become min(value, -1)."""
    raw = np.asarray(raw)
    img = raw.astype(np.float32)
    bad = raw == np.iinfo(raw.dtype).max
    if min_valid > 0:
        bad |= raw < min_valid
    if overload is not None:
        img[raw >= overload] = -2.0
    img[bad] = -1.0
    if mask is not None:
        m = ~np.asarray(mask, bool)
        img[m] = np.minimum(img[m], -1.0)
    return img


def replace_spec(spec, **kw):
    return replace(spec, **kw)


class DeviceSpots:
    """A sweep's spot table on the device for the frame generator, with per-bucket lists of the spots that reach
    each run of BUCKET frames (|z - zc| < 5 sigma_z), so that a wedge's spots are found without a scan of the
    table. The noise of a spot's pixels is keyed by the spot's index in the table and the frame: any partition of the
    frames into wedges renders the same frames."""

    BUCKET = 32

    def __init__(self, spec: SweepSpec, table, device="cuda"):
        import torch
        self.spec = spec
        g = spec.geometry()
        self.t = {k: torch.as_tensor(np.ascontiguousarray(table[k], np.float64)).to(device)
                  for k in ("x", "y", "z", "counts", "sig_t", "sig_r", "sig_z")}
        z, sz = np.asarray(table["z"], float), np.asarray(table["sig_z"], float)
        lo = np.floor((z - 5 * sz) / self.BUCKET).astype(np.int64)      # frame index f covers z in [f, f + 1)
        hi = np.floor((z + 5 * sz) / self.BUCKET).astype(np.int64)
        n_b = int(np.ceil((spec.nframes + 1) / self.BUCKET)) + 1
        lo, hi = np.clip(lo, 0, n_b - 1), np.clip(hi, 0, n_b - 1)
        cnt = hi - lo + 1
        idx = np.repeat(np.arange(z.size, dtype=np.int32), cnt)
        bk = (np.repeat(lo, cnt) + (np.arange(idx.size) - np.repeat(np.cumsum(cnt) - cnt, cnt))).astype(np.int32)
        o = np.argsort(bk, kind="stable")
        self.idx = idx[o]
        self.start = np.searchsorted(bk[o], np.arange(n_b + 1))
        self.device = device
        self.bg = (spec.background, spec.ramp, float(g.orgx), float(g.orgy),
                   float(max(np.hypot(np.array([1.0, spec.nx, 1.0, spec.nx]) - g.orgx,
                                      np.array([1.0, 1.0, spec.ny, spec.ny]) - g.orgy).max(), 1.0)))
        self.org = (float(g.orgx), float(g.orgy))

    def spots_for(self, first_frame, n_frames):
        """Indices of the spots that reach frames first_frame..first_frame + n_frames - 1 (1-based)."""
        b0 = max((first_frame - 1) // self.BUCKET, 0)
        b1 = min((first_frame - 1 + n_frames - 1) // self.BUCKET, len(self.start) - 2)
        if b1 < b0:
            return np.zeros(0, np.int32)
        return np.unique(self.idx[self.start[b0]:self.start[b1 + 1]])

    def render(self, first_frame, n_frames, out, stream=None):
        """Frames first_frame .. first_frame + n_frames - 1 into the device int32 tensor out (n_frames, ny, nx)."""
        import ctypes as C

        from . import native as N
        from .device import h2d
        spec = self.spec
        idx = self.spots_for(first_frame, n_frames)
        it = h2d(idx, None, self.device) if idx.size else None
        sp = N.XiSynthSpots()
        sp.n = int(idx.size)
        sp.index = N.ptr(it)
        for k, v in self.t.items():
            setattr(sp, k, N.ptr(v))
        sp.orgx, sp.orgy = self.org
        bg = N.XiSynthBackground()
        bg.level, bg.ramp, bg.orgx, bg.orgy, bg.rmax = self.bg
        rc = N.load().xi_synth_frames(C.byref(sp), C.byref(bg), int(first_frame), int(n_frames), spec.ny, spec.nx,
                                      int(spec.seed), 1 if spec.gaps else 0, N.ptr(out), N.stream_handle(stream))
        if rc != 0:
            raise RuntimeError("xi_synth_frames: " + N.load().xi_synth_last_error().decode())
        return out


def device_frames(spec: SweepSpec, table, first_frame, n_frames, out=None, device="cuda", stream=None, spots=None):
    """Frames first_frame .. first_frame + n_frames - 1 rendered on the device (int32 view of uint32 counts),
    shape (n_frames, ny, nx). Same model as `render_frames`, with a device counter-based Poisson draw (so the pixel
    values differ from the host generator's). `spots`: a DeviceSpots of the table (made here when not given)."""
    import torch

    from . import native as N
    N.require_cuda()
    if out is None:
        out = torch.empty((n_frames, spec.ny, spec.nx), dtype=torch.int32, device=device)
    if spots is None:
        spots = DeviceSpots(spec, table, device)
    return spots.render(first_frame, n_frames, out, stream)
