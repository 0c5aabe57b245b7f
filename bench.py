#!/usr/bin/env python
"""Benchmark of the B200 shoebox integration (drop-in for XPG's INTEGRATE stage).

Workload (default `config2-block`): one 360-frame phi block of the 16M-pixel sweep (4148 x 4362 px of 75 um at
120 mm, lambda 0.98 A, 0.1 deg frames, P 21 21 21 60/85/120 A, sigma_M 0.15 deg, sigma_D 0.03 deg, background 0.2,
5 x 5 profile regions). A step is one full `integrate()` call of the drop-in API on that block: predictions and shoebox
plan, frame gather, pass 1, profile learning, adaptive widths, pass 2, results back on the host. The block's frames
(every frame its boxes reach) are synthetic, seeded and rendered on the device before timing (`data`); the frame
stack (~34 GB) is far larger than L2, so no flush is needed between steps.

  value  reflections integrated per second with the frames resident in HBM (device-timed, CUDA events, max over
         ranks), whole job over all ranks;
  e2e    the same with the frames in pinned host memory, uploaded inside every step (the transfer thread sends
         each 2-frame chunk raw or packed to one byte a pixel on the host's cores, whichever keeps the link busy;
         h2d_bytes_per_step counts the bytes that crossed);
  roofline  of the dominant kernel (largest share of device time): algorithmic bytes per launch / live CUDA-event
         launch duration, against the measured HBM copy bandwidth;
  cpu_baseline  the oracle (numpy restatement of the reference's CPU path) on a bounded sample of the same block.

With --gpus N (torchrun, one rank per GPU) every rank integrates a block of its own sweep (replicas: sweeps are
independent; weak scaling). `--impl reference` times the CPU restatement of the reference on all host cores.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "integrated reflections/s (one 360-frame phi block of the 16M-pixel sweep per step)"
UNIT = "refl/s"


def _env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons: started before the workload's set-up (its start-up load
    stays out of the timed steps), summarised over the samples taken between mark() and stop() (the timed region)."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.gpu = gpu_index
        self.p = None
        self.t0 = None

    def mark(self):
        self.t0 = time.time()

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t1 = time.time()
        self.p.terminate()
        self.p.wait(5)
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        timed = []
        for r in rows:
            try:
                ts = datetime.datetime.strptime(r[0].strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except (ValueError, IndexError):
                continue
            if self.t0 is None or self.t0 <= ts <= t1:
                timed.append(r)
        rows = timed or rows
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "0x1", "1"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def reduce_over_ranks(t, n, dist=None, device="cuda"):
    """Whole-job timing of replicas: the slowest rank's time and the total units over all ranks."""
    if dist is None:
        return t, n
    import torch
    tt = torch.tensor([t], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    nn = torch.tensor([float(n)], device=device, dtype=torch.float64)
    dist.all_reduce(nn)
    return float(tt.item()), int(nn.item())


def replica_seed(workload, rank):
    """Seed of the sweep a rank integrates: replicas integrate independent sweeps (different crystal orientation
    and noise), so no data is exchanged between ranks."""
    return (2 if workload.startswith("config2") else 1) + rank


class Block:
    """One phi block of a synthetic sweep, planned and rendered on the device."""

    def __init__(self, name, seed_offset=0, device="cuda"):
        from xpg_b200 import synth
        from xpg_b200.plan import IntegrationModel, plan_integration
        seed = replica_seed(name, seed_offset)
        if name == "config2-block":
            self.spec = synth.config2(seed=seed)
            self.edges = np.array([0.0, 360.0])
        elif name == "config2-small":          # a 20-frame block of the same sweep (profiling captures)
            self.spec = synth.config2(seed=seed)
            self.edges = np.array([0.0, 20.0])
        elif name == "config1":
            self.spec = synth.config1(seed=seed)
            self.edges = np.array([0.0, 100.0])
        else:
            raise ValueError(name)
        s = self.spec
        self.exp = s.experiment()
        self.dmin = s.resolution_limit()
        self.model = IntegrationModel(sigma_d=s.sigma_d, sigma_m=s.sigma_m)
        # frames the block's boxes reach
        probe = plan_integration([self.exp], self.edges, self.model, self.dmin, 1e9, (1, s.nframes), 0.05,
                                 s.n_regions_xy, True, True)
        self.n_frames = int(min(max(probe.need_hi) + 1, s.nframes))
        self.plan = plan_integration([self.exp], self.edges, self.model, self.dmin, 1e9, (1, self.n_frames), 0.05,
                                     s.n_regions_xy, True, True)
        self.n_refl = self.plan.n
        _, self.table = synth.reflection_table(s, z_range=(-5.0, self.n_frames + 5.0))
        self.frames = synth.device_frames(s, self.table, 1, self.n_frames, device=device)
        self.device = device

    def integrate(self, frames):
        from xpg_b200.integrate import integrate
        return integrate(frames, [self.exp], self.edges, self.model, self.dmin, frames=(1, self.n_frames),
                         verbose=False, n_regions_xy=self.spec.n_regions_xy)

    def source(self, host=None):
        from xpg_b200.frames import U32Frames
        return U32Frames(self.frames if host is None else host, first=1, overload=self.spec.overload,
                         device=self.device)

    def bytes_per_kernel(self):
        """Algorithmic bytes of every kernel over one step: each shoebox voxel read once (4 B), the per-pixel and
        per-frame tables written or read once, the row's scalars; the gather reads every raw pixel its boxes cover
        and writes the box once; decode_bins reads and writes the binned rows."""
        p = self.plan
        V = (p.Dz * p.bx * p.bx).astype(np.float64)
        P = (p.bx * p.bx).astype(np.float64)
        raw = (np.minimum(p.Dz * p.fb, np.maximum(self.n_frames - p.iz0, 0)) * (p.bx * p.pxs) ** 2).astype(np.float64)
        return {"pass1": float((4 * V + 17 * P + 4 * p.Dz + 92).sum()),
                "pass2": float((4 * V + 12 * P + 52).sum()),
                "gather": float((4 * raw + 4 * V).sum()),
                "decode_bins": float((8 * V * (p.fb > 1)).sum())}


SAMPLE = dict(a=100, wz=24, crop=1024)     # frame window and detector crop of the CPU sample

# DRAM bytes (read + write) per shoebox voxel of the pass kernels, from one ncu capture of a launch of the same
# kernels on the config-2 geometry (a 20-frame block, `--workload config2-small`: the 2,597-reflection launch of
# 31 x 31 x 33 boxes, 82.4 M voxels); the traffic of a launch here is that figure times its voxels
DRAM_BYTES_PER_VOXEL = {"pass1": 4.554, "pass2": 4.439}


def _sample_rows(p, nx, ny):
    """Rows of the CPU sample: boxes inside frames [a, a + wz) and inside a crop x crop detector patch."""
    a, wz, c = SAMPLE["a"], SAMPLE["wz"], SAMPLE["crop"]
    x0, y0 = nx // 2 + 300, ny // 2 + 300
    x0, y0 = min(x0, nx - c), min(y0, ny - c)
    inside = (p.iz0 >= a) & (p.iz0 + p.Dz * p.fb <= a + wz) & (p.pxs == 1) & \
        (p.ix0 >= x0) & (p.ix0 + p.bx <= x0 + c) & (p.iy0 >= y0) & (p.iy0 + p.bx <= y0 + c)
    return np.flatnonzero(inside), (y0, x0)


def _frame_prep_seconds(raw_full, overload):
    """Host time to prepare one full frame (encoding and mask ceiling, as XPG's frame loop does for every frame)."""
    from oracle import gather as OG
    ts = []
    for f in raw_full:
        t0 = time.perf_counter()
        OG.prepare_frame(f, overload, 0, None)
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts))


def _cpu_baseline(blk, budget_s=20.0, max_rows=400):
    """The oracle restatement of the reference's CPU path on a bounded sample of the block, 1 core: gather, pass 1
    and pass 2 of sample rows timed directly, plus each reflection's share of the full-frame preparation (one frame
    timed, charged as frames / reflections of the block)."""
    from oracle import kernels as OK
    from oracle import pipeline as OP
    p = blk.plan
    s = blk.spec
    a, wz, c = SAMPLE["a"], SAMPLE["wz"], SAMPLE["crop"]
    rows, (y0, x0) = _sample_rows(p, s.nx, s.ny)
    rows = rows[:max_rows]
    full = blk.frames[a:a + 3].cpu().numpy().view(np.uint32)
    t_prep = _frame_prep_seconds(full, s.overload)
    raw = blk.frames[a:a + wz, y0:y0 + c, x0:x0 + c].cpu().numpy().view(np.uint32)
    prep = OP.prepared_frames(raw, a, s.overload, [1])
    g = blk.exp.geom
    det = OK.detector_consts(g, None)
    prof = np.repeat(OK.gaussian_profile()[None], p.nreg, 0)
    prof = prof / (prof.sum(axis=(1, 2), keepdims=True) * (9.0 / 40) ** 2)
    t0 = time.perf_counter()
    done = 0
    for k in range(0, rows.size, 20):
        OP.integrate_rows(prep, list(range(a, a + wz)), OP.row_payload(p, rows[k:k + 20]), det,
                          g.s0.astype(np.float32), g.axis.astype(np.float32), np.float32(np.radians(g.z_to_phi(0.0))),
                          np.float32(np.radians(g.osc)), np.radians(s.sigma_d), np.radians(s.sigma_m), 1.0,
                          OK.rc_default_weights(), prof, origin=(y0, x0))
        done = k + min(20, rows.size - k)
        if time.perf_counter() - t0 > budget_s:
            break
    t_rows = time.perf_counter() - t0
    per_refl = t_rows / max(done, 1) + t_prep * blk.n_frames / blk.n_refl
    return {"value": round(1.0 / per_refl, 2), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{done} reflections of the block (boxes inside frames {a + 1}-{a + wz}): gather, pass 1 and "
                      f"pass 2 by the numpy oracle in {t_rows:.1f} s, plus the block's full-frame preparation "
                      f"({t_prep * 1e3:.0f} ms per frame x {blk.n_frames} frames) shared over its {blk.n_refl} "
                      f"reflections"}


def _parity(blk, res, n_min=500):
    """Post-check of the timed run's results (after the timed region): a stratified sample of the block's rows
    (every shoebox shape group) integrated again by the CPU restatement from the same raw frames with the block's
    learnt profiles and adapted widths; worst error per key relative to max(|value|, scale) (tests/tolerance.py),
    and the rows outside tolerance per key (integers: rows that differ)."""
    from oracle.blockcheck import check_rows, stratified_rows
    p, s = blk.plan, blk.spec
    rows = stratified_rows(p, np.arange(p.n), n_min=n_min)

    def crop(f0, f1, y0, y1, x0, x1):
        return blk.frames[f0:f1, y0:y1, x0:x1].cpu().numpy().view(np.uint32)
    t0 = time.perf_counter()
    worst, bad, info = check_rows(crop, p, rows, res, 0, blk.exp.geom, blk.n_frames, s.ny, s.nx, s.overload,
                                  blk.model.gain)
    return dict(info, worst={k: float(f"{v:.3g}") for k, v in worst.items()}, outside_tolerance=bad,
                seconds=round(time.perf_counter() - t0, 1))


def run(args):
    import torch
    rank, world, local = _env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from xpg_b200 import device as D
    from xpg_b200.csrc import build
    if build.stale():
        build.build()
    clocks = Clocks(local)
    clocks.start()                # before the set-up: nvidia-smi's start-up load stays out of the timed steps
    blk = Block(args.workload, seed_offset=rank)
    src = blk.source()
    res = None
    for _ in range(args.warmup):  # results held across calls as in the timed loop: the pinned result buffers that
        res = blk.integrate(src)  # two live results need are allocated here, not in a timed step
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    D.TIMER.reset()
    D.TIMER.enabled = True
    clocks.mark()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    n_ok = 0
    marks = []
    for _ in range(args.steps):
        res = blk.integrate(src)
        n_ok += int(np.isfinite(res.refl["iprf"]).sum())
        marks.append(torch.cuda.Event(enable_timing=True))
        marks[-1].record()
    e1.record()
    torch.cuda.synchronize()
    D.TIMER.enabled = False
    clk = clocks.stop()
    res_timed = res
    t = e0.elapsed_time(e1) * 1e-3
    step_ms = [round(a.elapsed_time(b), 1) for a, b in zip([e0] + marks[:-1], marks)]
    ksum = D.TIMER.summary()
    launches = D.TIMER.launches
    t_max, n_total = reduce_over_ranks(t, blk.n_refl * args.steps, dist)
    value = n_total / t_max
    # roofline of the dominant kernel
    peak, peak_kind = _peaks()
    bpk = blk.bytes_per_kernel()
    dom = max(ksum, key=lambda k: ksum[k][1]) if ksum else None
    roof = None
    if dom is not None:
        n_l, t_k = ksum[dom]
        per_launch = bpk.get(dom, 0.0) * args.steps / max(n_l, 1)
        achieved = per_launch / (t_k / n_l) / 1e9
        vox = float((blk.plan.Dz * blk.plan.bx.astype(np.float64) ** 2).sum()) * args.steps / max(n_l, 1)
        traffic = round(DRAM_BYTES_PER_VOXEL[dom] * vox / 1e9, 3) if dom in DRAM_BYTES_PER_VOXEL else None
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_unit": "GB per launch",
                "algorithmic": round(per_launch / 1e9, 3), "peak_kind": peak_kind,
                "launches": n_l, "ms_per_launch": round(t_k / n_l * 1e3, 4),
                "share": {k: round(v[1] / max(sum(x[1] for x in ksum.values()), 1e-12), 4) for k, v in ksum.items()},
                "ms_per_step": {k: round(v[1] / args.steps * 1e3, 2) for k, v in ksum.items()}}
    # end to end: frames from pinned host memory, uploaded inside every step; results read back by the API
    e2e = None
    if not args.no_e2e:
        host = torch.empty(blk.frames.shape, dtype=torch.int32, pin_memory=True)
        host.copy_(blk.frames)
        hsrc = blk.source(host)
        res = blk.integrate(hsrc)
        res = blk.integrate(hsrc)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        k2 = max(1, min(args.steps, args.e2e_steps))
        moved0 = dict(hsrc.transfer)
        f0.record()
        for _ in range(k2):
            res = blk.integrate(hsrc)
        f1.record()
        torch.cuda.synchronize()
        te, _ = reduce_over_ranks(f0.elapsed_time(f1) * 1e-3, 0, dist)
        n_out = sum(v.nbytes for v in res.refl.values() if isinstance(v, np.ndarray))
        moved = {k: (hsrc.transfer.get(k, 0) - moved0.get(k, 0)) / k2 for k in ("h2d_bytes", "chunks_raw",
                                                                                 "chunks_packed")}
        e2e = {"value": round(blk.n_refl * world * k2 / te, 1), "unit": UNIT,
               "h2d_bytes_per_step": int(moved["h2d_bytes"]), "d2h_bytes_per_step": int(n_out), "steps": k2,
               "frame_bytes_per_step": int(host.numel() * 4),
               "chunks_per_step": {"raw": moved["chunks_raw"], "packed": moved["chunks_packed"]}}
        del host
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = _cpu_baseline(blk)
    parity = None
    if rank == 0 and not args.no_parity:
        parity = _parity(blk, res_timed)
    if dist is not None:
        dist.barrier()
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(t_max / args.steps * 1e3, 3), "step_ms": step_ms,
                "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 accumulation)",
                "data": "synthetic: seeded 16M-pixel frames rendered on the device (spec in xpg_b200/synth.py)",
                "config": {"workload": args.workload, "reflections_per_step": blk.n_refl,
                           "frames_per_step": blk.n_frames, "detector": [blk.spec.nx, blk.spec.ny],
                           "voxels_per_step": int((blk.plan.Dz * blk.plan.bx ** 2).sum()),
                           "l2": "inputs larger than L2 (frame stack ~{:.0f} GB)".format(blk.frames.numel() * 4 / 1e9),
                           "parallelism": f"replicas x{world} (one block per rank)"},
                "integrated_per_step": n_ok // max(args.steps, 1),
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
                "parity": parity}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


_REF = {}


def _ref_init(prep, a, wz, spec_d, nreg, origin):
    """Worker set-up (spawned process, once per pool): the prepared frame crops and the block constants."""
    from oracle import kernels as OK
    from xpg_b200 import synth
    spec = synth.SweepSpec(**spec_d)
    g = spec.geometry()
    prof = np.repeat(OK.gaussian_profile()[None], nreg, 0)
    _REF.update(prep=prep, a=a, wz=wz, spec=spec, g=g, det=OK.detector_consts(g, None), origin=origin,
                prof=prof / (prof.sum(axis=(1, 2), keepdims=True) * (9.0 / 40) ** 2))


def _ref_worker(payload):
    """Oracle work of one chunk of rows: gather, pass 1, pass 2 from the worker's prepared frame crops."""
    from oracle import kernels as OK
    from oracle import pipeline as OP
    r = _REF
    g, spec = r["g"], r["spec"]
    OP.integrate_rows(r["prep"], list(range(r["a"], r["a"] + r["wz"])), payload, r["det"], g.s0.astype(np.float32),
                      g.axis.astype(np.float32), np.float32(np.radians(g.z_to_phi(0.0))), np.float32(np.radians(g.osc)),
                      np.radians(spec.sigma_d), np.radians(spec.sigma_m), 1.0, OK.rc_default_weights(), r["prof"],
                      origin=r["origin"])
    return len(payload)


def reference_arm(args):
    """The reference's CPU path (its numpy restatement in oracle/) on all host cores: per step a bounded sample of
    the block's reflections (gather, pass 1, pass 2 spread over spawned processes) plus their share of the block's
    full-frame preparation (one frame timed per step, frames spread over the cores as XPG's decode pool does)."""
    rank, world, local = _env()
    if rank != 0:
        return
    import multiprocessing as mp
    from dataclasses import asdict

    import torch
    from oracle import pipeline as OP
    from oracle.plan import plan_integration
    from xpg_b200 import synth
    from xpg_b200.plan import IntegrationModel
    cores = len(os.sched_getaffinity(0))
    spec = synth.config2() if args.workload == "config2-block" else synth.config1()
    edges = np.array([0.0, 360.0]) if args.workload == "config2-block" else np.array([0.0, 100.0])
    exp = spec.experiment()
    model = IntegrationModel(spec.sigma_d, spec.sigma_m)
    dmin = spec.resolution_limit()
    probe = plan_integration([exp], edges, model, dmin, 1e9, (1, spec.nframes), 0.05, spec.n_regions_xy, True, True)
    n_frames = int(min(max(probe.need_hi) + 1, spec.nframes))
    p = plan_integration([exp], edges, model, dmin, 1e9, (1, n_frames), 0.05, spec.n_regions_xy, True, True)
    a, wz, c = SAMPLE["a"], SAMPLE["wz"], SAMPLE["crop"]
    rows_all, (y0, x0) = _sample_rows(p, spec.nx, spec.ny)
    _, table = synth.reflection_table(spec, z_range=(a - 40.0, a + wz + 40.0))
    if torch.cuda.is_available():
        raw = synth.device_frames(spec, table, a + 1, wz).cpu().numpy().view(np.uint32)
    else:
        raw = synth.render_frames(spec, range(a + 1, a + wz + 1), table)
    prep = OP.prepared_frames(raw[:, y0:y0 + c, x0:x0 + c], a, spec.overload, [1])
    per_step = max(cores * 24, 48)
    sd = asdict(spec)
    sd.pop("U", None)
    ctx = mp.get_context("spawn")
    n_done, t_all = 0, 0.0
    with ctx.Pool(cores, initializer=_ref_init, initargs=(prep, a, wz, sd, p.nreg, (y0, x0))) as pool:
        def step(k):
            lo = (k * per_step) % max(rows_all.size - per_step, 1)
            rows = rows_all[lo:lo + per_step]
            chunks = [OP.row_payload(p, rows[i::cores]) for i in range(cores)]
            t0 = time.perf_counter()
            n = sum(pool.map(_ref_worker, [ch for ch in chunks if ch]))
            t_rows = time.perf_counter() - t0
            t_prep = _frame_prep_seconds(raw[:1], spec.overload)
            return n, t_rows + t_prep * n_frames / p.n * n / cores
        for k in range(args.warmup):
            step(k)
        for k in range(args.steps):
            n, t = step(args.warmup + k)
            n_done += n
            t_all += t
    value = n_done / t_all
    line = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_all / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 accumulation)", "impl": "reference",
            "data": "synthetic: seeded 16M-pixel frames (spec in xpg_b200/synth.py)",
            "config": {"workload": args.workload, "reflections_per_step": per_step},
            "cpu_baseline": {"value": round(value, 2), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{per_step} reflections per step of the block (boxes inside frames "
                                       f"{a + 1}-{a + wz}, a {c} px detector patch): gather + pass 1 + pass 2 by the "
                                       f"numpy restatement over {cores} spawned processes, plus their share of the "
                                       f"block's full-frame preparation"},
            "e2e": {"value": round(value, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def decode_bench(args):
    """The bitshuffle-LZ4 frame decode (Eiger chunks): the LZ4 stage on the host's cores (xi_bslz4_lz4_stage) and the
    bit unshuffle on the device (xi_bitunshuffle), each timed alone, printed as one JSON line. The chunk is the
    committed fixture tests/golden/bslz4_band.bin (a 256 x 4148 band of a config-2 frame: Poisson background 0.2,
    seed 11, flagged columns; made by tests/golden/make_bslz4_band.py); the band is regenerated here from its seed and
    the decode checked against it before timing. The unshuffle runs on full 4148 x 4362 frames."""
    import ctypes as C

    import torch
    from xpg_b200 import native
    from xpg_b200.csrc import build
    if build.stale():
        build.build()
    lib = native.load()
    ny, nx = 256, 4148
    rng = np.random.default_rng(11)
    band = rng.poisson(0.2, (ny, nx)).astype(np.uint32)
    band[:, ::259] = 0xFFFFFFFF
    chunk = np.fromfile(ROOT / "tests" / "golden" / "bslz4_band.bin", np.uint8)
    out = torch.empty(band.nbytes, dtype=torch.uint8).pin_memory()
    nb, be = C.c_int64(), C.c_int64()
    call = lambda: lib.xi_bslz4_lz4_stage(chunk.ctypes.data, chunk.size, 4, C.c_void_p(out.data_ptr()), band.nbytes,
                                          0, C.byref(nb), C.byref(be))
    native.check(call(), "xi_bslz4_lz4_stage")
    n = 4148 * 4362
    dev_in = out.cuda()
    chk = torch.empty(band.size, dtype=torch.int32, device="cuda")
    native.check(lib.xi_bitunshuffle(native.ptr(dev_in), band.size, 4, be.value, native.ptr(chk),
                                     native.stream_handle()), "xi_bitunshuffle")
    if not np.array_equal(chk.cpu().numpy().view(np.uint32), band.reshape(-1)):
        raise RuntimeError("decoded band differs from the band")
    k = max(args.steps, 1) * 40
    t0 = time.perf_counter()
    for _ in range(k):
        call()
    th = (time.perf_counter() - t0) / k
    staged = torch.randint(0, 256, (n * 4,), dtype=torch.uint8, device="cuda")
    frame = torch.empty(n, dtype=torch.int32, device="cuda")
    st = native.stream_handle()
    go = lambda: lib.xi_bitunshuffle(native.ptr(staged), n, 4, 2048, native.ptr(frame), st)
    for _ in range(max(args.warmup, 3)):
        native.check(go(), "xi_bitunshuffle")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kd = max(args.steps, 1) * 4
    e0.record()
    for _ in range(kd):
        go()
    e1.record()
    torch.cuda.synchronize()
    td = e0.elapsed_time(e1) * 1e-3 / kd
    peak, peak_kind = _peaks()
    dev_gbs = 8.0 * n / td / 1e9
    print(json.dumps({
        "metric": "bitshuffle-LZ4 frame decode (Eiger chunks)", "unit": "GB/s of uint32 frame bytes",
        "compression_ratio": round(band.nbytes / chunk.size, 2),
        "host_lz4_stage": {"value": round(band.nbytes / th / 1e9, 2),
                           "frames_per_s_16M": round(band.nbytes / th / (4 * n), 1),
                           "cores": len(os.sched_getaffinity(0)),
                           "sample": f"{ny} x {nx} uint32 band, {chunk.size} B chunk, {k} calls"},
        "device_unshuffle": {"value": round(4.0 * n / td / 1e9, 1), "ms_per_16M_frame": round(td * 1e3, 3),
                             "roofline": {"bound": "hbm", "achieved": round(dev_gbs, 1), "peak": peak, "unit": "GB/s",
                                          "frac": round(dev_gbs / peak, 4), "peak_kind": peak_kind, "traffic": None,
                                          "algorithmic": "4 B read + 4 B written per pixel"}},
    }), flush=True)


def spots_bench(args):
    """The strong-pixel classifier of spot finding (both passes) on 4148 x 4362 float32 frames (Poisson background 0.2,
    flagged columns, 3000 spots per frame), timed with CUDA events, one JSON line; cpu_baseline: the oracle's numpy
    restatement of XPG's classifier on one frame, one core."""
    import torch
    from xpg_b200.csrc import build
    from xpg_b200.spotfind import make_finder
    if build.stale():
        build.build()
    rng = np.random.default_rng(3)
    nb, ny, nx = 8, 4362, 4148
    img = rng.poisson(0.2, (nb, ny, nx)).astype(np.float32)
    img[:, :, ::259] = -1.0
    for f in range(nb):
        ys, xs = rng.integers(5, ny - 5, 3000), rng.integers(5, nx - 5, 3000)
        for y, x in zip(ys, xs):
            img[f, y - 1:y + 2, x - 1:x + 2] += rng.integers(5, 200)
    dev = torch.from_numpy(img).cuda()
    find = make_finder()
    for _ in range(max(args.warmup, 3)):
        find(dev, 1.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        s, m = find(dev, 1.0)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / args.steps
    px = nb * ny * nx
    # algorithmic bytes: the frame read by both passes and the background pass (12 B), the first-pass mask and mean
    # written and read (2 x 5 B), the background flags (2 B), the outputs (5 B), the uint8 -> bool copy (2 B)
    alg = 31.0 * px
    peak, peak_kind = _peaks()
    t0 = time.perf_counter()
    from oracle import spotfind as OS
    OS.find(img[:1], 1.0)
    tc = time.perf_counter() - t0
    print(json.dumps({
        "metric": "spot-finding strong-pixel classifier", "unit": "frames/s (4148 x 4362 px)",
        "value": round(nb / t, 1), "ms_per_frame": round(t / nb * 1e3, 3), "frames_per_call": nb,
        "roofline": {"bound": "hbm", "achieved": round(alg / t / 1e9, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(alg / t / 1e9 / peak, 4), "peak_kind": peak_kind, "traffic": None,
                     "algorithmic": "31 B per pixel over the three launches and the mask copy"},
        "cpu_baseline": {"value": round(1.0 / tc, 3), "unit": "frames/s", "cores": 1, "kind": "port",
                         "sample": "one frame through the oracle's numpy restatement of XPG's classifier"},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--workload", default="config2-block", choices=("config2-block", "config2-small", "config1"))
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the post-check of the results against the oracle")
    ap.add_argument("--decode", action="store_true", help="time the bitshuffle-LZ4 frame decode instead")
    ap.add_argument("--spots", action="store_true", help="time the spot-finding classifier instead")
    args = ap.parse_args()
    if args.decode:
        decode_bench(args)
    elif args.spots:
        spots_bench(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
