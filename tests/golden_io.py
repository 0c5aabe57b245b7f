"""Loading of the golden fixtures (reference outputs on seeded sweeps) for the tests."""
from __future__ import annotations

import json
import zlib
from functools import lru_cache
from pathlib import Path

import numpy as np

from xpg_b200 import synth

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("config1", "adaptive", "superpix", "binned", "crowded", "precision", "foreign")


@lru_cache(maxsize=None)
def load(name):
    z = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    return {k: z[k] for k in z.files}


def spec_of(name):
    d = json.loads(str(load(name)["spec_json"]))
    d["cell"] = tuple(d["cell"])
    d["beam"] = tuple(d["beam"])
    d["axis"] = tuple(d["axis"])
    return synth.SweepSpec(**d)


def kwargs_of(name):
    return json.loads(str(load(name)["kw_json"]))


def template(spec):
    ys, xs = np.mgrid[0:spec.ny, 0:spec.nx]
    return (1.0 + 0.35 * np.sin(xs / 37.0) * np.cos(ys / 53.0)).astype(np.float32)


def static_mask(spec):
    m = np.ones((spec.ny, spec.nx), bool)
    m[spec.ny // 3: spec.ny // 3 + 9, spec.nx // 4: spec.nx // 2] = False
    return m


def foreign_of(name):
    """The foreign-spot list (x, y, z) a case was integrated with, or None (same seeded list as the generator's)."""
    if not kwargs_of(name).get("foreign"):
        return None
    spec = spec_of(name)
    rng = np.random.default_rng(21)
    n = 2400
    return (rng.uniform(1.0, spec.nx, n), rng.uniform(1.0, spec.ny, n), rng.uniform(0.0, spec.nframes, n))


def case_inputs(name):
    """(spec, template or None, mask or None, exclude_frames) of a case."""
    spec = spec_of(name)
    kw = kwargs_of(name)
    return (spec, template(spec) if kw.get("template") else None, static_mask(spec) if kw.get("mask") else None,
            tuple(kw.get("exclude_frames", ())))


@lru_cache(maxsize=2)
def frames_of(name):
    """The case's uint32 frames, re-rendered and checked against the fixture's per-frame crc32."""
    spec = spec_of(name)
    fr = synth.render_frames(spec)
    crc = np.array([zlib.crc32(f.tobytes()) for f in fr], np.uint32)
    want = load(name)["frames_crc"]
    if not np.array_equal(crc, want):
        raise AssertionError(f"{name}: rendered frames differ from the fixture's (generator drift)")
    return fr


def chunks(name):
    """Indices of the kernel-call chunks stored in a fixture."""
    z = load(name)
    return sorted(int(k[1:].split("_")[0]) for k in z if k.startswith("c") and k.endswith("_shape"))


def chunk(name, i):
    z = load(name)
    p = f"c{i}_"
    d = {k[len(p):]: v for k, v in z.items() if k.startswith(p)}
    rc = {k[3:]: v for k, v in d.items() if k.startswith("rc_")}
    nb = {k[3:]: v for k, v in d.items() if k.startswith("nb_")}
    o1 = {k[3:]: v for k, v in d.items() if k.startswith("o1_")}
    o2 = {k[3:]: v for k, v in d.items() if k.startswith("o2_")}
    return d, rc, nb, o1, o2


def row_dict(rc, j):
    """Per-reflection inputs of row j of a chunk as plain scalars."""
    r = dict(S=np.asarray(rc["S"][j], np.float32), phi=np.float32(rc["phi"][j]), ix0=int(rc["ix0"][j]),
             iy0=int(rc["iy0"][j]), iz0=int(rc["iz0"][j]), fb=np.float32(rc["fb"][j]), region=int(rc["region"][j]),
             has_p=np.float32(rc["has_p"][j]), pS=np.asarray(rc["pS"][j], np.float32),
             pphi=np.float32(rc["pphi"][j]))
    if "pxs" in rc:
        r["pxs"] = int(rc["pxs"][j])
    return r


def nb_row(nb, j):
    return {k: np.asarray(v[j], np.float32) for k, v in nb.items()}
