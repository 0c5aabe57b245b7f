"""Generate the golden fixtures of the integration path by running XPG's own `integrate()` on seeded synthetic
sweeps, in this container (the reference is importable from its checkout; it does not exist where the GPU tests
run, so the fixtures are committed).

Reference settings (they make every result independent of how reflections are batched):
* `integrate_kernels.IRLS_TOL = 0`: always N_IRLS = 6 profile-fit iterations (`xpg/integrate_kernels.py:19-22`);
* XPG_DECODE_PROCS=0, XPG_GATHER_PROCESS=0: frames decoded and gathered in the calling process;
* `integrate.lattice_allowed` replaced by the centring rule (it imports gemmi, which is absent here).

Frames come from `xpg_b200.synth.render_frames` (seeded, reproducible frame by frame) through an in-memory subclass
of XPG's `ImageSet` whose `_read_native` returns the uint32 frame and its 0xFFFFFFFF flags, i.e. the reference's
own Eiger encoding path (`xpg/io/images.py:72-102`, `:408-419`).

Each fixture `<case>.npz` holds
* `spec_json`: the sweep spec and integrate() arguments (the GPU tests re-render the frames from it);
* `frames_crc`: crc32 of every rendered frame (guards against generator drift);
* `out_<key>`: the reference's per-reflection results (`IntegrationResult.refl`), `prof_<b>` the learnt profiles,
  `bp_json` the per-block parameters;
* `c<i>_*`: per kernel call (one chunk of one shoebox shape): the shoebox chunk `sb` for up to ROWS_KEEP rows, the
  per-row inputs (`rc_*`, `nb_*`), the scalars, the detector constants, and the outputs of pass 1, the profile
  accumulation (num / den of the block) and pass 2.

Run from the repository root:  python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import json
import os
import sys
import time
import zlib
from dataclasses import asdict
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

os.environ.setdefault("XPG_DECODE_PROCS", "0")
os.environ.setdefault("XPG_GATHER_PROCESS", "0")
os.environ.setdefault("XPG_GATHER_THREADS", "4")
os.environ.setdefault("XPG_DEVICE", "cpu")

from xpg_b200 import synth  # noqa: E402

ROWS_KEEP = 48          # shoebox rows kept per kernel call (the sb arrays dominate the fixture size)


def _cases():
    """name -> (spec, integrate kwargs)."""
    c = {}
    c["config1"] = (synth.config1(), dict())
    # bright spots, two phi blocks: profile learning, the adaptive sigma_M / rocking-curve / sigma_D update
    c["adaptive"] = (synth.config1(name="adaptive", nframes=60, block_frames=30, mean_i0=3000.0, seed=5,
                                   hot_fraction=0.004), dict())
    # super-pixels (spot sigma of several pixels) with a background template and a static mask
    c["superpix"] = (synth.SweepSpec(name="superpix", nx=420, ny=400, qx=0.075, distance=200.0, wavelength=1.0,
                                     osc=0.2, nframes=24, cell=(150.0, 150.0, 150.0, 90, 90, 90),
                                     space_group="P 21 21 21", sigma_d=0.085, sigma_m=0.15, mean_i0=800.0,
                                     background=1.0, seed=7, dmin=2.2, gaps=False, sensor_thickness=0.45, mu=3.4),
                     dict(template=True, mask=True))
    # wide rocking curves: phi-binned shoeboxes (fb > 1), excluded frames, frames missing at the sweep ends
    c["binned"] = (synth.SweepSpec(name="binned", nx=260, ny=270, qx=0.172, distance=90.0, wavelength=1.0,
                                   osc=0.1, nframes=110, cell=(60.0, 70.0, 80.0, 90, 90, 90), space_group="P 21 21 21",
                                   sigma_d=0.04, sigma_m=0.45, mean_i0=600.0, background=0.7, seed=8, dmin=2.6,
                                   gaps=False, hot_fraction=0.01),
                   dict(exclude_frames=(40, 41)))
    # crowded: large C-centred cell, overlapping partners (joint fit), many neighbours
    c["crowded"] = (synth.SweepSpec(name="crowded", nx=300, ny=310, qx=0.172, distance=70.0, wavelength=1.0,
                                    osc=0.3, nframes=24, cell=(230.0, 180.0, 210.0, 90.0, 101.0, 90.0),
                                    space_group="C 1 2 1", sigma_d=0.05, sigma_m=0.2, mean_i0=300.0, background=0.6,
                                    seed=9, dmin=3.5, gaps=True),
                    dict())
    # config 3's error model on a small sweep: weak reflections and shoeboxes > 40% masked
    c["precision"] = (synth.config1(name="precision", nframes=40, weak_fraction=0.05, dead_fraction=0.02, seed=3),
                      dict())
    # spots of another crystal given as foreign_spots: masked like non-modelled neighbours (extra neighbour columns)
    c["foreign"] = (synth.config1(name="foreign", nframes=40, seed=6), dict(foreign=True))
    # spot-width estimation (moments-only integrate calls on sub-ranges)
    c["sigmas"] = (synth.config1(name="sigmas", nframes=60, mean_i0=2000.0, seed=4), dict(estimate=True))
    return c


def _ref_modules():
    from refpath import import_reference
    import_reference()
    import xpg.integrate as RI
    import xpg.integrate_kernels as RK
    from xpg.geometry import Geometry as RGeometry
    from xpg.io.images import ImageSet
    from xpg.models import Crystal as RCrystal, Experiment as RExperiment
    from xpg_b200.geometry import centring_allowed
    RK.IRLS_TOL = 0.0
    RI.lattice_allowed = centring_allowed
    return RI, RK, RGeometry, RCrystal, RExperiment, ImageSet


def _ref_experiment(spec, RGeometry, RCrystal, RExperiment):
    g = spec.geometry()
    rg = RGeometry(wavelength=g.wavelength, beam=g.beam, axis=g.axis, orgx=g.orgx, orgy=g.orgy,
                   distance=g.distance, ed1=g.ed1, ed2=g.ed2, qx=g.qx, qy=g.qy, nx=g.nx, ny=g.ny, phi0=g.phi0,
                   osc=g.osc, starting_frame=g.starting_frame, polarization_fraction=g.polarization_fraction,
                   polarization_normal=g.polarization_normal, sensor_thickness=g.sensor_thickness, mu=g.mu)
    rc = RCrystal(U=spec.orientation(), cell=np.array(spec.cell, float), space_group=spec.space_group)
    return RExperiment(rg, rc)


def foreign_spots(spec, n=2400, seed=21):
    """Spot positions of a foreign crystal (x, y in pixels, z in frames), seeded: uniform over the detector and the
    sweep, so that many fall within a reflection's neighbour reach and some within 2.5 sigma of its centre."""
    rng = np.random.default_rng(seed)
    return (rng.uniform(1.0, spec.nx, n), rng.uniform(1.0, spec.ny, n), rng.uniform(0.0, spec.nframes, n))


def _template(spec):
    """A smooth background template (relative scale ~0.7-1.4) for the template case."""
    ys, xs = np.mgrid[0:spec.ny, 0:spec.nx]
    t = 1.0 + 0.35 * np.sin(xs / 37.0) * np.cos(ys / 53.0)
    return t.astype(np.float32)


def _static_mask(spec):
    m = np.ones((spec.ny, spec.nx), bool)
    m[spec.ny // 3: spec.ny // 3 + 9, spec.nx // 4: spec.nx // 2] = False      # a beam-stop arm
    return m


def run_case(name, spec, kw, out_dir=HERE):
    RI, RK, RGeometry, RCrystal, RExperiment, ImageSet = _ref_modules()
    t0 = time.time()
    frames = synth.render_frames(spec)
    crc = np.array([zlib.crc32(f.tobytes()) for f in frames], np.uint32)

    class MemImages(ImageSet):
        def __init__(self):
            super().__init__(min_valid=0.0, overload=spec.overload)
            self.nx, self.ny, self.first, self.last = spec.nx, spec.ny, 1, spec.nframes

        def _read_native(self, frame):
            raw = frames[frame - 1]
            return raw, raw == np.iinfo(raw.dtype).max

    exp = _ref_experiment(spec, RGeometry, RCrystal, RExperiment)
    g = exp.geom
    edges = spec.block_edges()
    blocks = [exp] * (len(edges) - 1)
    model = RI.IntegrationModel(sigma_d=spec.sigma_d, sigma_m=spec.sigma_m, gain=1.0)
    dmin = spec.resolution_limit()
    tmpl = _template(spec) if kw.get("template") else None
    mask = _static_mask(spec) if kw.get("mask") else None
    args = dict(frames=(1, spec.nframes), mask=mask, minimum_zeta=0.05, verbose=False,
                n_regions_xy=spec.n_regions_xy, exclude_frames=tuple(kw.get("exclude_frames", ())),
                bkg_template=tmpl)
    if kw.get("foreign"):
        args["foreign_spots"] = foreign_spots(spec)
    calls = []
    orig = RK.make_kernels

    def wrapped_make_kernels(Dz, Dy, Dx, n_regions, G=RK.PROFILE_GRID):
        p1, acc, p2 = orig(Dz, Dy, Dx, n_regions, G)

        def w1(sb, rc, det, axis, s0, frames_phi0, osc, sd, sm, gain, prof, nb, rcw):
            r = p1(sb, rc, det, axis, s0, frames_phi0, osc, sd, sm, gain, prof, nb, rcw)
            calls.append(dict(kind="p1", shape=(Dz, Dy, Dx), sb=_np(sb), rc={k: _np(v) for k, v in rc.items()},
                              nb={k: _np(v) for k, v in nb.items()}, det=det,
                              scal=dict(frames_phi0=float(frames_phi0), osc=float(osc), sd=float(sd), sm=float(sm),
                                        gain=float(gain)), axis=_np(axis), s0=_np(s0), rcw=_np(rcw),
                              out={k: _np(v) for k, v in r.items() if k != "_h"}, res=r))
            return r

        def wacc(img2, ok2, J, u1, u2, region, isum, sel, seff):
            num, den = acc(img2, ok2, J, u1, u2, region, isum, sel, seff)
            calls.append(dict(kind="acc", shape=(Dz, Dy, Dx), inputs=dict(img2=_np(img2), ok2=_np(ok2), J=_np(J),
                              u1=_np(u1), u2=_np(u2), region=_np(region), isum=_np(isum), seff=_np(seff)),
                              num=_np(num), den=_np(den)))
            return num, den

        def w2(sb, rc, det, axis, s0, frames_phi0, osc, sd, sm, gain, prof, bg, nbm_x, nb, rcw, pix=None):
            r = p2(sb, rc, det, axis, s0, frames_phi0, osc, sd, sm, gain, prof, bg, nbm_x, nb, rcw, pix)
            calls.append(dict(kind="p2", shape=(Dz, Dy, Dx), prof=_np(prof), bg=_np(bg), nbg=_np(nbm_x),
                              scal=dict(sd=float(sd), sm=float(sm), gain=float(gain)), rcw=_np(rcw),
                              out={k: _np(v) for k, v in r.items() if k != "_h"}))
            return r
        return w1, wacc, w2

    RI.make_kernels = wrapped_make_kernels
    RK._KERNEL_CACHE.clear()
    RI._KERNEL_CACHE.clear()
    try:
        if kw.get("estimate"):
            res_model = RI.estimate_sigmas(MemImages(), exp, model, max(dmin, 2.0), (1, spec.nframes), verbose=False,
                                           bkg_template=tmpl)
            res = None
        else:
            res = RI.integrate(MemImages(), blocks, edges, model, dmin, **args)
    finally:
        RI.make_kernels = orig
        RK._KERNEL_CACHE.clear()
        RI._KERNEL_CACHE.clear()
    t_ref = time.time() - t0

    save = dict(spec_json=json.dumps(_spec_dict(spec)), kw_json=json.dumps({k: v for k, v in kw.items()}),
                frames_crc=crc, dmin=np.float64(dmin), edges=edges, t_ref=np.float64(t_ref))
    det0 = None
    if res is not None:
        for k, v in res.refl.items():
            save["out_" + k] = np.asarray(v)
        for b, p in res.profiles.items():
            save[f"prof_{b}"] = np.asarray(p, np.float32)
        save["bp_json"] = json.dumps({str(k): v for k, v in getattr(res, "block_params", {}).items()})
    else:
        save["model"] = np.array([res_model.sigma_d, res_model.sigma_m], np.float64)
        save["history"] = np.array(getattr(res_model, "history", []), np.float64)
    # kernel calls: each pass-1 call (one chunk of one shoebox shape) with the pass-2 call of the same chunk (the
    # i-th pass-2 call of a block fits the block's i-th pass-1 chunk), and every profile accumulation
    chunks, block_p1, cur, seen_p2 = [], [], [], False
    for c in calls:
        if c["kind"] == "p1":
            if seen_p2:
                cur, seen_p2 = [], False
            cur.append(len(chunks))
            chunks.append(dict(p1=c, p2=None))
        elif c["kind"] == "p2":
            if not seen_p2:
                block_p1, seen_p2, k2 = list(cur), True, 0
            chunks[block_p1[k2]]["p2"] = c
            k2 += 1
    lim = 8 if not kw.get("estimate") else 3
    for i, ch in enumerate(chunks[:lim]):
        c = ch["p1"]
        p = f"c{i}_"
        save[p + "shape"] = np.array(c["shape"], np.int32)
        m = c["sb"].shape[0]
        rows = _pick_rows(c, m)
        save[p + "rows"] = rows
        save[p + "sb"] = c["sb"][rows]
        for k, v in c["rc"].items():
            save[p + "rc_" + k] = v[rows]
        for k, v in c["nb"].items():
            save[p + "nb_" + k] = v[rows]
        for k, v in c["scal"].items():
            save[p + k] = np.float64(v)
        save[p + "axis"], save[p + "s0"], save[p + "rcw"] = c["axis"], c["s0"], c["rcw"]
        for k, v in c["out"].items():
            save[p + "o1_" + k] = v[rows]
        if det0 is None:
            det0 = c["det"]
        c2 = ch["p2"]
        if c2 is not None:
            save[p + "prof"] = c2["prof"]
            for k, v in c2["scal"].items():
                save[p + "p2_" + k] = np.float64(v)
            save[p + "p2_rcw"] = c2["rcw"]
            for k, v in c2["out"].items():
                save[p + "o2_" + k] = v[rows]
    accs = [c for c in calls if c["kind"] == "acc"]
    for i, c in enumerate(accs[:4]):
        p = f"a{i}_"
        save[p + "shape"] = np.array(c["shape"], np.int32)
        save[p + "num"], save[p + "den"] = c["num"], c["den"]
        for k, v in c["inputs"].items():
            save[p + "in_" + k] = v
    if det0 is not None:
        for k, v in det0.items():
            save["det_" + k] = _np(v) if hasattr(v, "shape") else np.float64(v)
    if tmpl is not None:
        save["template_used"] = np.array(True)
    if mask is not None:
        save["mask_used"] = np.array(True)
    path = out_dir / f"{name}.npz"
    np.savez_compressed(path, **save)
    n = len(res.refl["x"]) if res is not None else -1
    print(f"{name}: {n} reflections, {len(calls)} kernel calls, reference {t_ref:.1f}s, "
          f"{path.stat().st_size / 1e6:.2f} MB")
    return path


def _pick_rows(c, m):
    """Rows kept from a kernel call: partners, binned, overloaded, masked and neighbour-affected rows first, then
    the rest in order, up to ROWS_KEEP."""
    out = c["out"]
    pri = np.zeros(m)
    rc = c["rc"]
    pri += 4 * (np.asarray(rc["has_p"]) > 0.5)
    pri += 3 * (np.asarray(rc["fb"]) > 1)
    pri += 2 * (np.asarray(out["n_over"]) > 0)
    pri += 2 * (np.asarray(out["n_fg_masked"]) > 0)
    pri += 1 * (np.asarray(out["n_fg_nb"]) > 0)
    order = np.argsort(-pri, kind="stable")
    return np.sort(order[:ROWS_KEEP]).astype(np.int64)


def _np(v):
    import torch
    if torch.is_tensor(v):
        return v.detach().cpu().numpy()
    return np.asarray(v)


def _spec_dict(spec):
    d = asdict(spec)
    d.pop("U", None)
    return d


if __name__ == "__main__":
    cases = _cases()
    names = sys.argv[1:] or list(cases)
    for n in names:
        s, kw = cases[n]
        run_case(n, s, kw)
