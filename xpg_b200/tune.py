"""Autotuner of the pass launches: which box sides share a persistent launch (the size bins) and the CTA shape.

A batched launch sizes its shared memory, threads per CTA and staging for the largest box of its bin: wide bins
put small boxes in CTAs sized for large ones (fewer resident CTAs), narrow bins make more launches (more tails). The
CTA shape of large boxes (128 threads at 6 CTAs per SM, or 256 at 3), the largest box staged in shared memory by
a bulk copy, and pass 2's fit-list capacity (the fitted voxels kept in shared memory for its six IRLS iterations;
a row with more fits from the box each time) trade resident reflections per SM against work per CTA. The tuner
times pass 1 and pass 2 of real blocks for launch shapes, then list capacities, then candidate bin edges (subsets of
the box-side buckets present, at most `max_bins` bins), and keeps the fastest; results are stored per device name in `tuned.json` beside this file, which the library applies
when it loads (`native.load`) and `device.batched_items` reads.

    python -m xpg_b200.tune [--workload config4|config2] [--max-bins 4]      (on the GPU)
"""
from __future__ import annotations

import itertools
import json
from pathlib import Path

import numpy as np
import torch

from . import device as D

TUNED = Path(__file__).resolve().parent / "tuned.json"
XY_BUCKETS = (9, 13, 17, 23, 31, 41, 55, 73, 97)


def candidates(sides, max_bins=4):
    """Bin edge tuples over the box sides present: the largest side always closes the last bin."""
    present = sorted(set(int(s) for s in sides))
    top = present[-1]
    inner = present[:-1]
    out = []
    for k in range(0, max_bins):
        for c in itertools.combinations(inner, k):
            out.append(tuple(c) + (top,))
    return out


def _time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3


SHAPES = ({"wide_threads": 256, "pass1_stage_bytes": 48 * 1024}, {"wide_threads": 128, "pass1_stage_bytes": 48 * 1024},
          {"wide_threads": 256, "pass1_stage_bytes": 0}, {"wide_threads": 128, "pass1_stage_bytes": 0},
          {"wide_threads": 128, "pass1_stage_bytes": 96 * 1024})


LIST_CAPS = (2048, 4096, 8192, 12288, 16384)
CAP_DEFAULTS = {"pass2_list_cap": 2048, "pass2_list_cap_large": 8192}


def _apply(shape):
    """Sets a launch shape, the list capacities it does not name at their defaults."""
    from . import native as N
    N.tune(**dict(CAP_DEFAULTS, **shape))


def tune_round(picks, max_bins=4, reps=3, device="cuda", shapes=SHAPES, caps=LIST_CAPS):
    """Times the candidate launch shapes, then pass 2's fit-list capacities, then bin sets on one batched round of
    completed blocks. picks: list of (SweepRun, block) whose pass 1 and learning are done (their set entries valid).
    Returns [(seconds, bins, shape)] fastest first."""
    from . import native as N
    sets1, sets2, groups = [], [], []
    for k, (run, b) in enumerate(picks):
        blk = run.live[b]
        rs = blk.rowset
        det = run.detector(run.exp_blocks[b].geom)
        sets1.append(D.rowset_entry(det, rs, blk.c1[3], blk.arena, blk.p1))
        sets2.append(D.rowset_entry(det, rs, blk.c2[0], blk.arena, blk.p1, blk.prof, blk.p2))
        groups.append((k, np.arange(rs.n), rs.bx, rs.Dz))
    t1, t2 = D.RowSetTable(sets1, device), D.RowSetTable(sets2, device)
    sides = np.concatenate([g[2] for g in groups])
    out = []
    base = candidates(sides, 1)[0]
    for shape in shapes:                 # launch shape first, on one bin of all sides
        _apply(shape)
        launches = D.batched_items(groups, base, device)
        out.append((_time(lambda: (D.pass1_batched(t1, launches), D.pass2_batched(t2, launches)), reps), base, shape))
    best_shape = dict(min(out, key=lambda r: r[0])[2])
    _apply(best_shape)
    for key in ("pass2_list_cap", "pass2_list_cap_large"):   # pass 2's fit-list capacities (small, large boxes)
        for cap in caps:
            shape = dict(best_shape, **{key: cap})
            _apply(shape)
            launches = D.batched_items(groups, base, device)
            out.append((_time(lambda: (D.pass1_batched(t1, launches), D.pass2_batched(t2, launches)), reps), base,
                        shape))
        best_shape = dict(min(out, key=lambda r: r[0])[2])
        _apply(best_shape)
    for bins in candidates(sides, max_bins)[1:]:
        launches = D.batched_items(groups, bins, device)
        t = _time(lambda: (D.pass1_batched(t1, launches), D.pass2_batched(t2, launches)), reps)
        out.append((t, bins, best_shape))
    out.sort(key=lambda r: r[0])
    return out


def save(device_name, table, workload):
    data = json.loads(TUNED.read_text()) if TUNED.exists() else {}
    t, bins, shape = table[0]
    data[device_name] = {"bins": list(bins), "shape": shape, "workload": workload,
                         "measured": [{"seconds": round(t_, 5), "bins": list(b), "shape": sh}
                                      for t_, b, sh in table[:16]]}
    TUNED.write_text(json.dumps(data, indent=1) + "\n")


def load_shape(device_name=None):
    """Tuned launch shape of this device (xi_tune arguments), or None."""
    if not TUNED.exists():
        return None
    try:
        name = device_name or torch.cuda.get_device_name()
    except Exception:
        return None
    entry = json.loads(TUNED.read_text()).get(name)
    return entry.get("shape") if entry else None


def load_bins(device_name=None):
    """Tuned bins of this device (None when not tuned)."""
    if not TUNED.exists():
        return None
    try:
        name = device_name or torch.cuda.get_device_name()
    except Exception:
        return None
    entry = json.loads(TUNED.read_text()).get(name)
    return tuple(entry["bins"]) if entry else None


def main():
    import argparse
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench
    from .batch import run_jobs  # noqa: F401
    from .integrate import SweepRun
    from . import synth
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="config4", choices=("config4", "config2"))
    ap.add_argument("--max-bins", type=int, default=4)
    args = ap.parse_args()
    specs = synth.config4() if args.workload == "config4" else [synth.config2(nframes=480)]
    jobs = bench._jobs_of(specs, bench.WEDGE_FRAMES)
    from . import memplan
    room = 0.9 * memplan.budget()
    runs = []
    for j in jobs:                        # up to 6 sweeps whose planned peaks fit the device together
        run = SweepRun(j.images, j.exp_blocks, j.block_edges, j.model, j.dmin, early_pass1=False, verbose=False,
                       mem_budget=room, **j.kwargs)
        if run.mem["peak"] > room or "passes" in run.mem or run.mem["parts"] > 1:
            run.close()
            continue
        room -= run.mem["peak"]
        runs.append(run)
        if len(runs) == 6:
            break
    picks = []
    for run in runs:                      # the first completed block of every sweep
        done = []
        for w in range(len(run.wedges)):
            done = run.feed(w)
            if done:
                break
        done = done or run.remaining()
        b = done[0]
        run.pass1_stage(b)
        run.learn(b)
        picks.append((run, b))
    table = tune_round(picks, args.max_bins)
    name = torch.cuda.get_device_name()
    save(name, table, args.workload)
    print(json.dumps({"device": name, "best": {"bins": list(table[0][1]), "shape": table[0][2]},
                      "seconds": round(table[0][0], 5), "worst": [round(table[-1][0], 5), list(table[-1][1]),
                                                                  table[-1][2]], "candidates": len(table),
                      "shapes": [{"seconds": round(t, 5), "shape": sh} for t, b, sh in table if len(b) == 1]}))
    for run in runs:
        run.close()


if __name__ == "__main__":
    main()
