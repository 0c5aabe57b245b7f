"""What XPG's INTEGRATE stage does with the integration's result after the path (`xpg/stage_integrate.py:408-447`):
the Lorentz-polarisation and absorption correction, the usable rows and their split by lattice, and the two files it
writes, `xpg_integrated.npz` and the legacy `INTEGRATE.HKL` (`xpg/io/legacy.py:71-100`, `:102-107`, `:140-182`).

Host code (numpy), O(n) over the reflections once the device results are on the host. It takes the geometry and
crystal of either package (attributes by name: `beam`, `axis`, `polarization_*`, `ed1..3`, `segments`, `cell`,
`Astar`, `space_group`, ...).
"""
from __future__ import annotations

import datetime

import numpy as np

from . import __version__

# Total mass attenuation coefficients of dry air (cm^2 / g) against photon energy (keV), NIST XCOM: the nodes XPG
# interpolates log-log for the air path between crystal and detector (`xpg/geometry.py:422-431`, `:434-446`).
AIR_DENSITY = 1.205e-3                    # g / cm^3
AIR_MU_RHO = ((5, 39.31), (6, 22.70), (8, 9.921), (10, 5.120), (15, 1.614), (20, 0.7779), (30, 0.3538),
              (40, 0.2485), (50, 0.2080), (60, 0.1875), (80, 0.1662), (100, 0.1541))
HC_KEV_A = 12.398419843320026             # photon energy (keV) x wavelength (A)


def air_mu(wavelength):
    """Linear attenuation coefficient of air (1/mm) at a wavelength (A)."""
    e = np.array([t[0] for t in AIR_MU_RHO], float)
    m = np.array([t[1] for t in AIR_MU_RHO], float)
    mu_rho = float(np.exp(np.interp(np.log(HC_KEV_A / wavelength), np.log(e), np.log(m))))
    return mu_rho * AIR_DENSITY / 10.0


def _unit(v):
    v = np.asarray(v, float)
    return v / np.linalg.norm(v)


def lp_factor(g, S):
    """(zeta, polarisation P) of diffracted wave vectors S (..., 3); intensities are corrected by |zeta| / P
    (`xpg/geometry.py:394-407`)."""
    e = S / np.linalg.norm(S, axis=-1, keepdims=True)
    e0 = np.asarray(g.beam, float)
    zeta = np.cross(e, e0) @ np.asarray(g.axis, float)
    pn = np.asarray(g.polarization_normal, float)
    n = pn - np.dot(pn, e0) * e0
    n = n / np.linalg.norm(n)
    emain = np.cross(n, e0)
    f = g.polarization_fraction
    return zeta, f * (1 - (e @ emain) ** 2) + (1 - f) * (1 - (e @ n) ** 2)


def absorption_factors(g, S, air=True):
    """Attenuation of the recorded intensity: sensor efficiency (when the sensor thickness and attenuation are known)
    times air transmission along the crystal-detector path (`xpg/geometry.py:372-392`). Segmented detectors take the
    normal and the path of the segment the ray hits."""
    e = S / np.linalg.norm(S, axis=-1, keepdims=True)
    f = np.ones(e.shape[:-1])
    ed3 = np.cross(_unit(g.ed1), _unit(g.ed2)) if not hasattr(g, "ed3") else np.asarray(g.ed3, float)
    segmented = bool(getattr(g, "segmented", False))
    if segmented:
        x, y = g.s_to_pixel(S)
        x, y = np.nan_to_num(x, nan=1.0), np.nan_to_num(y, nan=1.0)
        P0, Bx, By = g.panels()
        k = np.maximum(np.asarray(_segment_of(g, x, y), int), 0)
        cosn = np.einsum("...k,...k->...", e, np.cross(Bx[k] / g.qx, By[k] / g.qy))
    else:
        cosn = e @ ed3
    t, mu = float(getattr(g, "sensor_thickness", 0.0) or 0.0), float(getattr(g, "mu", 0.0) or 0.0)
    if t > 0 and mu > 0:
        f = f * -np.expm1(-mu * t / np.clip(cosn, 1e-3, 1.0))
    if air:
        if segmented:
            path = np.linalg.norm(g.pixel_to_lab(x, y), axis=-1)
        else:
            path = g.distance / np.clip(e @ ed3, 1e-3, 1.0)
        f = f * np.exp(-air_mu(g.wavelength) * path)
    return f


def _segment_of(g, x, y):
    for name in ("segment_of", "_segment_of"):
        fn = getattr(g, name, None)
        if fn is not None:
            return fn(x, y)
    return np.zeros(np.shape(x), int)


def _rows(refl, m):
    return {k: (v[m] if isinstance(v, np.ndarray) and v.shape[:1] == m.shape else v) for k, v in refl.items()}


def lp_correct(refl, g, air=True):
    """The stage's correction and selection (`xpg/stage_integrate.py:408-431`): rlp = |zeta| / P / absorption; I, sig
    (profile fitting) and Isum, sigsum (summation) times rlp; PEAK = 100 x the fitted profile fraction recorded x the
    box coverage; CORR in percent; rows with a finite I and a positive finite sigma kept, split by lattice.
    Returns (rows of lattice 0, {k - 1: rows of lattice k})."""
    refl = dict(refl)
    zeta, pol = lp_factor(g, np.asarray(refl["S"], float))
    rlp = np.abs(zeta) / pol / absorption_factors(g, np.asarray(refl["S"], float), air=air)
    refl["rlp"] = rlp
    refl["I"] = refl["iprf"] * rlp
    refl["sig"] = np.sqrt(np.maximum(refl["vprf"], 0)) * rlp
    refl["Isum"] = refl["isum"] * rlp
    refl["sigsum"] = np.sqrt(np.maximum(refl["vsum"], 0)) * rlp
    refl["peak"] = 100 * np.clip(refl["p_valid"] / np.maximum(refl["p_total"], 1e-9), 0, 1) * \
        refl.get("coverage", 1.0)
    refl["corr"] = 100 * np.nan_to_num(refl["corr"])
    good = np.isfinite(refl["I"]) & np.isfinite(refl["sig"]) & (refl["sig"] > 0)
    refl = _rows(refl, good)
    lat = refl.get("lattice", np.zeros(len(refl["I"]), int))
    extra = {k - 1: _rows(refl, lat == k) for k in range(1, int(lat.max()) + 1 if lat.size else 1)}
    return _rows(refl, lat == 0), extra


def write_integrated_npz(path, refl, threads=None):
    """`xpg_integrated.npz`: every per-reflection array of the corrected rows but the per-frame profiles fz, in the
    file numpy's `savez_compressed` writes (a zip of deflated `.npy` members, read back by `np.load`), its members
    compressed on `threads` host threads at once (zlib releases the interpreter lock)."""
    arrays = {k: v for k, v in refl.items() if isinstance(v, np.ndarray) and k != "fz"}
    _write_npz_parallel(path, arrays, threads)


def _npy_bytes(a):
    import io
    buf = io.BytesIO()
    np.lib.format.write_array(buf, np.asanyarray(a), allow_pickle=False)
    return buf.getvalue()


def _deflate(raw):
    import zlib
    c = zlib.compressobj(6, zlib.DEFLATED, -15)          # raw deflate, zipfile's default level
    return c.compress(raw) + c.flush(), zlib.crc32(raw) & 0xFFFFFFFF


def _write_npz_parallel(path, arrays, threads=None):
    """A zip of deflated .npy members (local headers, data, central directory: the PKWARE APPNOTE layout zipfile
    writes); members over 4 GiB, or a file over 4 GiB, go through numpy's own writer (zip64)."""
    import os
    import struct
    import time as _time
    from concurrent.futures import ThreadPoolExecutor
    names = list(arrays)
    raws = [_npy_bytes(arrays[k]) for k in names]
    if sum(len(r) for r in raws) >= 0xFFFFFFFF // 2:
        np.savez_compressed(path, **arrays)
        return
    n_th = threads or max(1, min(len(raws), (os.cpu_count() or 2) - 1))
    with ThreadPoolExecutor(n_th) as ex:
        packed = list(ex.map(_deflate, raws))
    t = _time.localtime()
    dtime = (t.tm_hour << 11) | (t.tm_min << 5) | (t.tm_sec // 2)
    ddate = ((t.tm_year - 1980) << 9) | (t.tm_mon << 5) | t.tm_mday
    central, off = [], 0
    with open(path, "wb") as f:
        for k, raw, (data, crc) in zip(names, raws, packed):
            name = (k + ".npy").encode()
            head = struct.pack("<IHHHHHIIIHH", 0x04034B50, 20, 0, 8, dtime, ddate, crc, len(data), len(raw),
                               len(name), 0)
            f.write(head)
            f.write(name)
            f.write(data)
            central.append(struct.pack("<IHHHHHHIIIHHHHHII", 0x02014B50, 20, 20, 0, 8, dtime, ddate, crc, len(data),
                                       len(raw), len(name), 0, 0, 0, 0, 0o600 << 16, off) + name)
            off += len(head) + len(name) + len(data)
        cd = b"".join(central)
        f.write(cd)
        f.write(struct.pack("<IHHHHIIH", 0x06054B50, 0, 0, len(names), len(names), len(cd), off, 0))


def _frame_safe(z):
    """A frame coordinate printed with one decimal stays in its frame (z in [n - 1, n) is frame n; printed as n.0 it
    would read as frame n + 1) (`xpg/io/legacy.py:102-106`)."""
    z = np.asarray(z, float)
    return np.minimum(z, np.floor(z) + 0.94)


def _space_group_number(symbol):
    try:
        import gemmi
        return gemmi.SpaceGroup(symbol).number if symbol else 1
    except Exception:                 # without gemmi XPG writes 1 as well
        return 1


def _header(g, cell, R, sgnum, data_range, sigma_m, sigma_d, template):
    """The XDS header records shared by XPG's legacy files (`xpg/io/legacy.py:71-100`)."""
    axis = np.asarray(g.axis, float)
    s0 = np.asarray(g.s0, float) * g.wavelength
    ed1, ed2 = np.asarray(g.ed1, float), np.asarray(g.ed2, float)
    pn = np.asarray(g.polarization_normal, float)
    return [
        f"!NAME_TEMPLATE_OF_DATA_FRAMES={template}",
        f"!DATA_RANGE={data_range[0]:8d}{data_range[1]:8d}",
        f"!ROTATION_AXIS={axis[0]:10.6f}{axis[1]:10.6f}{axis[2]:10.6f}",
        f"!OSCILLATION_RANGE={g.osc:10.6f}",
        f"!STARTING_ANGLE={g.phi0:10.3f}",
        f"!STARTING_FRAME={g.starting_frame:8d}",
        f"!SPACE_GROUP_NUMBER={sgnum:5d}",
        f"!UNIT_CELL_CONSTANTS={cell[0]:10.3f}{cell[1]:10.3f}{cell[2]:10.3f}{cell[3]:8.3f}{cell[4]:8.3f}{cell[5]:8.3f}",
        f"!UNIT_CELL_A-AXIS={R[0, 0]:10.3f}{R[0, 1]:10.3f}{R[0, 2]:10.3f}",
        f"!UNIT_CELL_B-AXIS={R[1, 0]:10.3f}{R[1, 1]:10.3f}{R[1, 2]:10.3f}",
        f"!UNIT_CELL_C-AXIS={R[2, 0]:10.3f}{R[2, 1]:10.3f}{R[2, 2]:10.3f}",
        f"!REFLECTING_RANGE_E.S.D.={sigma_m:10.3f}",
        f"!BEAM_DIVERGENCE_E.S.D.={sigma_d:10.3f}",
        f"!X-RAY_WAVELENGTH={g.wavelength:10.6f}",
        f"!INCIDENT_BEAM_DIRECTION={s0[0]:10.6f}{s0[1]:10.6f}{s0[2]:10.6f}",
        f"!FRACTION_OF_POLARIZATION={g.polarization_fraction:8.3f}",
        f"!POLARIZATION_PLANE_NORMAL={pn[0]:10.6f}{pn[1]:10.6f}{pn[2]:10.6f}",
        "!DETECTOR=PILATUS",
        f"!NX={g.nx:6d}  NY={g.ny:6d}    QX={g.qx:10.6f}  QY={g.qy:10.6f}",
        f"!ORGX={g.orgx:10.2f}  ORGY={g.orgy:10.2f}",
        f"!DETECTOR_DISTANCE={g.distance:10.3f}",
        f"!DIRECTION_OF_DETECTOR_X-AXIS={ed1[0]:10.5f}{ed1[1]:10.5f}{ed1[2]:10.5f}",
        f"!DIRECTION_OF_DETECTOR_Y-AXIS={ed2[0]:10.5f}{ed2[1]:10.5f}{ed2[2]:10.5f}",
    ]


def write_integrate_hkl(path, exp, refl, data_range, sigma_m, sigma_d, template=""):
    """`INTEGRATE.HKL` of the corrected rows (`xpg/io/legacy.py:140-182`): the XDS header, 21 free-format items per
    reflection (H K L, I, sigma, calculated and observed position, RLP, PEAK, CORR, the beam directions as
    spherical angles in the laboratory frame), `!END_OF_DATA`."""
    g, c = exp.geom, exp.crystal
    R = np.linalg.inv(c.Astar)
    head = ["!OUTPUT_FILE=INTEGRATE.HKL    DATE=" + datetime.date.today().strftime("%d-%b-%Y"),
            f"!Generated by xpg_b200 {__version__}"]
    head += _header(g, np.asarray(c.cell, float), R, _space_group_number(getattr(c, "space_group", None)),
                    data_range, sigma_m, sigma_d, template)
    head += ["!NUMBER_OF_ITEMS_IN_EACH_DATA_RECORD=21",
             "!H,K,L,IOBS,SIGMA,XCAL,YCAL,ZCAL,RLP,PEAK,CORR,MAXC,",
             "!             XOBS,YOBS,ZOBS,ALF0,BET0,ALF1,BET1,PSI,ISEG",
             "!Items are separated by a blank and can be read in free-format",
             "!END_OF_HEADER"]
    n = len(refl["I"])
    beam = np.asarray(g.beam, float)
    u0 = beam / np.linalg.norm(beam)
    alf0, bet0 = np.degrees(np.arctan2(u0[1], u0[0])), np.degrees(np.arccos(np.clip(u0[2], -1, 1)))
    if "S" in refl:
        u1 = np.asarray(refl["S"], float)
        u1 = u1 / np.linalg.norm(u1, axis=1, keepdims=True)
        alf1, bet1 = np.degrees(np.arctan2(u1[:, 1], u1[:, 0])), np.degrees(np.arccos(np.clip(u1[:, 2], -1, 1)))
    else:
        alf1 = bet1 = np.zeros(n)
    xo = np.where(np.isfinite(refl["xo"]), refl["xo"], refl["x"])
    yo = np.where(np.isfinite(refl["yo"]), refl["yo"], refl["y"])
    zo = _frame_safe(np.where(np.isfinite(refl["zo"]), refl["zo"], refl["z"]))
    zc = _frame_safe(refl["z"])
    body = _records(n, refl, zc, xo, yo, zo, alf0, bet0, alf1, bet1)
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode())
        f.write(body)
        f.write(b"!END_OF_DATA\n")


def _records(n, refl, zc, xo, yo, zo, alf0, bet0, alf1, bet1):
    """The data records, formatted by the library on the host's cores (xi_format_integrate_hkl)."""
    import ctypes as C
    from . import native as N
    f64 = lambda a: np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64), (n,)))
    cols = dict(hkl=np.ascontiguousarray(np.asarray(refl["hkl"], np.int64).reshape(n, 3)), I=f64(refl["I"]),
                sig=f64(refl["sig"]), x=f64(refl["x"]), y=f64(refl["y"]), zc=f64(zc), rlp=f64(refl["rlp"]),
                peak=f64(refl["peak"]), corr=np.ascontiguousarray(np.nan_to_num(np.asarray(refl["corr"], np.float64))
                                                                  .astype(np.int64)),
                xo=f64(xo), yo=f64(yo), zo=f64(zo), alf1=f64(alf1), bet1=f64(bet1))
    r = N.XiHklRows()
    r.n = n
    for k, v in cols.items():
        setattr(r, k, v.ctypes.data)
    r.alf0, r.bet0 = float(alf0), float(bet0)
    lib = N.load()
    need = C.c_int64()
    cap = 160 * n
    for _ in range(2):
        buf = np.empty(max(cap, 1), np.uint8)
        rc = lib.xi_format_integrate_hkl(C.byref(r), buf.ctypes.data, cap, 0, C.byref(need))
        if rc == N.XI_OK:
            return buf[:need.value].tobytes()
        if rc != N.XI_E_LIMIT:
            N.check(rc, "xi_format_integrate_hkl")
        cap = need.value
    N.check(rc, "xi_format_integrate_hkl")
