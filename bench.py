#!/usr/bin/env python
"""Benchmark of the B200 shoebox integration (drop-in for XPG's INTEGRATE stage).

Workload (default `config2-sweep`): the whole 16M-pixel sweep, 3600 frames of 4148 x 4362 px (75 um at 120 mm,
lambda 0.98 A, 0.1 deg frames, P 21 21 21 60/85/120 A, sigma_M 0.15 deg, sigma_D 0.03 deg, background 0.2, 5 x 5
profile regions), integrated in 10 phi blocks of 360 frames with the adapted widths carried from block to block. A
step is one full `integrate()` call of the drop-in API on the sweep: predictions and shoebox plan, frames streamed in
32-frame wedges, gather, pass 1, profile learning, adaptive widths, pass 2 of every block, results back on the host.
The frames are synthetic and seeded, rendered on the device before timing and kept in HBM in the library's packed
transfer encoding (one byte a pixel plus exception pairs, 65 GB for the 260 GB of uint32 frames), widened wedge by
wedge inside the timed region. Other workloads: `config2-block` (one 360-frame block, raw frames resident),
`config2-small` (20 frames, for profiling captures), `config1` (config 1's 100-frame sweep). Inputs are far larger
than L2, so no flush is needed between steps.

  value  reflections integrated per second with the frames resident in HBM (device-timed, CUDA events, max over
         ranks), whole job over all ranks; pixel_gbs = the path's algorithmic bytes (every uint32 frame pixel once,
         every voxel a second time, 32 outputs per reflection) per second, pixel_hbm_frac against the measured peak;
  e2e    the same through the same API with the frames in pinned host memory (the sweep: its packed store; a block:
         raw uint32, packed by the transfer thread where that keeps the link busy), uploaded inside every step;
  roofline  of the dominant kernel (largest share of device time): algorithmic bytes per launch / live CUDA-event
         launch duration, against the measured HBM copy bandwidth;
  parity  after the timed region: stratified samples of rows of the first and the middle block integrated again by
         the CPU restatement from the same frames, the worst error per result key;
  cpu_baseline  the restatement of the reference's CPU path on a bounded random sample of the same workload.

With --gpus N (torchrun, one rank per GPU) every rank integrates a sweep of its own (replicas: sweeps are
independent; weak scaling). `--impl reference` times the CPU restatement of the reference on all host cores, on the
same workload and config, without CUDA.
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

METRICS = {"config2-sweep": "integrated reflections/s (the 16M-pixel, 3600-frame sweep per step)",
           "config2-block": "integrated reflections/s (one 360-frame phi block of the 16M-pixel sweep per step)",
           "config2-small": "integrated reflections/s (a 20-frame phi block of the 16M-pixel sweep per step)",
           "config1": "integrated reflections/s (the 1M-pixel, 100-frame sweep of config 1 per step)"}
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


WEDGE_FRAMES = 32


def workload_geometry(name, seed_offset=0):
    """(spec, block edges, frames integrated) of a workload: the whole 3600-frame sweep (10 phi blocks of 360 frames),
    one 360-frame block of it with every frame its boxes reach, a 20-frame block (profiling captures), or config 1's
    100-frame sweep."""
    from xpg_b200 import synth
    seed = replica_seed(name, seed_offset)
    if name == "config2-sweep":
        s = synth.config2(seed=seed)
        return s, s.block_edges(), s.nframes
    if name in ("config2-block", "config2-small"):
        s = synth.config2(seed=seed)
        return s, np.array([0.0, 360.0 if name == "config2-block" else 20.0]), None
    if name == "config1":
        s = synth.config1(seed=seed)
        return s, np.array([0.0, 100.0]), s.nframes
    raise ValueError(name)


def plan_workload(name, seed_offset, plan_integration):
    """The workload's spec, edges, frame count and shoebox plan (the device planner for the GPU arm, the CPU
    restatement for the reference arm: the same integers)."""
    from xpg_b200.plan import IntegrationModel
    s, edges, n_frames = workload_geometry(name, seed_offset)
    exp = s.experiment()
    model = IntegrationModel(sigma_d=s.sigma_d, sigma_m=s.sigma_m)
    args = (edges, model, s.resolution_limit(), 1e9)
    nb = len(edges) - 1
    if n_frames is None:                      # a block: every frame its boxes reach
        probe = plan_integration([exp] * nb, *args, (1, s.nframes), 0.05, s.n_regions_xy, True, True)
        n_frames = int(min(max(probe.need_hi) + 1, s.nframes))
    plan = plan_integration([exp] * nb, *args, (1, n_frames), 0.05, s.n_regions_xy, True, True)
    return s, exp, model, edges, n_frames, plan


def workload_config(name, spec, edges, n_frames, plan, world):
    """The `config` object of the bench line (the same for both arms)."""
    P = spec.nx * spec.ny
    return {"workload": name, "reflections_per_step": int(plan.n), "frames_per_step": int(n_frames),
            "phi_blocks": len(edges) - 1, "detector": [spec.nx, spec.ny],
            "voxels_per_step": int((plan.Dz * plan.bx.astype(np.int64) ** 2).sum()),
            "l2": f"inputs larger than L2 (frame stack {4 * P * n_frames / 1e9:.3g} GB of uint32)",
            "parallelism": f"replicas x{world} (one sweep per rank)"}


def alg_bytes(spec, n_frames, plan):
    """Algorithmic bytes of a step of the path: every uint32 frame pixel read once, every shoebox voxel read a second
    time by pass 2, 32 float64 outputs per reflection."""
    V = float((plan.Dz * plan.bx.astype(np.float64) ** 2).sum())
    return 4.0 * spec.nx * spec.ny * n_frames + 4.0 * V + 8.0 * 32 * plan.n


def bytes_per_kernel(plan, n_frames):
    """Algorithmic bytes of every kernel over one step: each shoebox voxel read once (4 B), the per-pixel and
    per-frame tables written or read once, the row's scalars; the gather reads every raw pixel its boxes cover and
    writes the box once; decode_bins reads and writes the binned rows; the unpack reads a packed byte and writes a
    uint32 per frame pixel."""
    p = plan
    V = (p.Dz * p.bx * p.bx).astype(np.float64)
    P = (p.bx * p.bx).astype(np.float64)
    raw = (np.minimum(p.Dz * p.fb, np.maximum(n_frames - p.iz0, 0)) * (p.bx * p.pxs) ** 2).astype(np.float64)
    return {"pass1": float((4 * V + 17 * P + 4 * p.Dz + 92).sum()),
            "pass2": float((4 * V + 12 * P + 52).sum()),
            "gather": float((4 * raw + 4 * V).sum()),
            "decode_bins": float((8 * V * (p.fb > 1)).sum())}


class Workload:
    """A workload on the device: its plan, its frames (resident in HBM: raw uint32 for a block, the whole sweep in
    the packed transfer encoding), and the same frames in pinned host memory for the end-to-end run."""

    def __init__(self, name, seed_offset=0, device="cuda"):
        import torch
        from xpg_b200 import synth
        from xpg_b200.plan import plan_integration
        self.name, self.device = name, device
        self.overlap = os.environ.get("XPG_BENCH_OVERLAP", "1") == "1"      # gathers on a stream of their own
        (self.spec, self.exp, self.model, self.edges, self.n_frames,
         self.plan) = plan_workload(name, seed_offset, plan_integration)
        s = self.spec
        _, self.table = synth.reflection_table(s, z_range=(-5.0, self.n_frames + 5.0))
        self.frames = self.store = self.dev_store = None
        if name == "config2-sweep":
            from xpg_b200 import frames as FR

            def render(k, n, out):
                synth.device_frames(s, self.table, k + 1, n, out=out, device=device)
            self.store = FR.pack_generated(render, self.n_frames, s.ny, s.nx, wedge=WEDGE_FRAMES, device=device)
            self.dev_store = self.store.to(device)
            self._tmp = torch.empty((s.ny, s.nx), dtype=torch.int32, device=device)
        else:
            self.frames = synth.device_frames(s, self.table, 1, self.n_frames, device=device)
        self.n_refl = self.plan.n

    def integrate(self, frames):
        from xpg_b200.integrate import integrate
        nb = len(self.edges) - 1
        return integrate(frames, [self.exp] * nb, self.edges, self.model, self.spec.resolution_limit(),
                         frames=(1, self.n_frames), verbose=False, n_regions_xy=self.spec.n_regions_xy,
                         wedge_frames=WEDGE_FRAMES, overlap=self.overlap)

    def source(self):
        """Frames resident in HBM."""
        from xpg_b200.frames import PackedFrames, U32Frames
        if self.dev_store is not None:
            return PackedFrames(self.dev_store, first=1, overload=self.spec.overload, device=self.device)
        return U32Frames(self.frames, first=1, overload=self.spec.overload, device=self.device)

    def host_source(self):
        """The same frames in pinned host memory (the sweep: its packed store; a block: raw uint32)."""
        import torch
        from xpg_b200.frames import PackedFrames, U32Frames
        if self.store is not None:
            return PackedFrames(self.store, first=1, overload=self.spec.overload, device=self.device, depth=12)
        host = torch.empty(self.frames.shape, dtype=torch.int32, pin_memory=True)
        host.copy_(self.frames)
        return U32Frames(host, first=1, overload=self.spec.overload, device=self.device)

    def drop_resident(self):
        """Frees the HBM copy of the sweep's packed frames (the end-to-end run reads the host copy)."""
        import torch
        if self.dev_store is not None:
            self.dev_store = None
            torch.cuda.empty_cache()

    def crop(self, f0, f1, y0, y1, x0, x1):
        """uint32 window [y0, y1) x [x0, x1) of frames f0..f1-1 (0-based) on the host."""
        import torch
        if self.frames is not None:
            return self.frames[f0:f1, y0:y1, x0:x1].cpu().numpy().view(np.uint32)
        out = np.empty((f1 - f0, y1 - y0, x1 - x0), np.uint32)
        for k in range(f0, f1):
            self.dev_store.unpack(k, self._tmp, torch.cuda.current_stream())
            out[k - f0] = self._tmp[y0:y1, x0:x1].cpu().numpy().view(np.uint32)
        return out

    def frame_bytes_on_host(self):
        return self.store.nbytes if self.store is not None else 4 * self.spec.nx * self.spec.ny * self.n_frames


# DRAM bytes (read + write) per shoebox voxel of the pass kernels, from one ncu capture of a launch of the same
# kernels on the config-2 geometry (a 20-frame block, `--workload config2-small`: the 2,597-reflection launch of
# 31 x 31 x 33 boxes, 82.4 M voxels); the traffic of a launch here is that figure times its voxels
DRAM_BYTES_PER_VOXEL = {"pass1": 5.060, "pass2": 4.432}


def _parity(wl, res, n_min=500):
    """Post-check of a timed run's results (after the timed region): stratified samples of rows (every shoebox shape
    group) of the first block and, for a sweep, of its middle block (widths carried over from the blocks before),
    integrated again by the CPU restatement from the same raw frames with each block's learnt profiles and adapted
    widths; worst error per key relative to max(|value|, scale) (tests/tolerance.py), and the rows outside tolerance
    per key (integers: rows that differ)."""
    from oracle.blockcheck import check_rows, stratified_rows
    p, s = getattr(res, "plan", wl.plan), wl.spec          # the plan integrated (blocks in parts if memory was short)
    nb = len(p.blocks_refl)
    blocks = sorted({0, nb // 2})
    t0 = time.perf_counter()
    worst, bad, rows_n, fitted = {}, {}, 0, 0
    for b in blocks:
        rows = stratified_rows(p, p.blocks_refl[b], n_min=n_min // len(blocks), seed=b)
        w, k, info = check_rows(wl.crop, p, rows, res, b, wl.exp.geom, wl.n_frames, s.ny, s.nx, s.overload,
                                wl.model.gain)
        for key, v in w.items():
            worst[key] = max(worst.get(key, 0.0), v)
        for key, v in k.items():
            bad[key] = bad.get(key, 0) + v
        rows_n += info["rows"]
        fitted += info["rows_fitted"]
    return dict(rows=rows_n, rows_fitted=fitted, blocks=blocks,
                worst={k: float(f"{v:.3g}") for k, v in worst.items()}, outside_tolerance=bad,
                seconds=round(time.perf_counter() - t0, 1))


def _frame_prep_seconds(raw_full, overload):
    """Host time to prepare one full frame (encoding and mask ceiling, as XPG's frame loop does for every frame)."""
    from oracle import gather as OG
    ts = []
    for f in raw_full:
        t0 = time.perf_counter()
        OG.prepare_frame(f, overload, 0, None)
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts))


def random_rows(plan, n, seed=0):
    """A uniform random sample of n rows (the workload's mix of shoebox shapes in proportion), sorted."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(plan.n, min(n, plan.n), replace=False))


def row_work(prep, payload, consts):
    """The restatement's work on rows whose box frames are prepared: gather, pass 1 and pass 2 (the CPU path of
    XPG for those reflections; default widths and the Gaussian prior profile, which do not change the work)."""
    from oracle import gather as OG
    from oracle import kernels as OK
    det, s0, axis, phi0, osc, sd, sm, rcw, prof = consts
    vox = 0
    for (r, nb), (frames, (oy, ox)) in zip(payload, prep):
        sb = OG.gather_shoebox(frames, sorted(frames), r["iz0"], r["fbi"], r["Dz"], r["bx"], r["iy0"] - oy,
                               r["ix0"] - ox)
        o1 = OK.pass1(sb, r, nb, det, s0, axis, phi0, osc, sd, sm, 1.0, rcw)
        pix = dict(zeta=o1["zeta"], J=o1["J"], u1=o1["u1"], u2=o1["u2"], seff=o1["seff"])
        OK.pass2(sb, r, nb, det, s0, axis, phi0, osc, sd, sm, 1.0, prof, o1["bg"], o1["nbg"], rcw, pix)
        vox += sb.size
    return len(payload), vox


def row_consts(spec, geom, nreg):
    from oracle import kernels as OK
    prof = np.repeat(OK.gaussian_profile()[None], nreg, 0)
    prof = prof / (prof.sum(axis=(1, 2), keepdims=True) * (9.0 / 40) ** 2)
    return (OK.detector_consts(geom, None), geom.s0.astype(np.float32), geom.axis.astype(np.float32),
            np.float32(np.radians(geom.z_to_phi(0.0))), np.float32(np.radians(geom.osc)), np.radians(spec.sigma_d),
            np.radians(spec.sigma_m), OK.rc_default_weights(), prof)


def prepared_boxes(crop, plan, rows, n_frames, ny, nx, overload):
    """Per row: its box frames prepared as XPG's frame loop prepares them, and the window origin."""
    from oracle.blockcheck import _box_frames
    return [_box_frames(crop, plan, j, n_frames, ny, nx, overload) for j in rows]


def _cpu_baseline(wl, budget_s=20.0, n_rows=400):
    """The restatement of the reference's CPU path on a bounded sample of the workload, 1 core: gather, pass 1 and
    pass 2 of a uniform random sample of its rows timed directly, plus each reflection's share of the full-frame
    preparation (one frame timed, charged as frames / reflections)."""
    from oracle.pipeline import row_payload
    p, s = wl.plan, wl.spec
    rows = random_rows(p, n_rows, seed=7)
    prep = prepared_boxes(wl.crop, p, rows, wl.n_frames, s.ny, s.nx, s.overload)
    full = wl.crop(0, 3, 0, s.ny, 0, s.nx)
    t_prep = _frame_prep_seconds(full, s.overload)
    consts = row_consts(s, wl.exp.geom, p.nreg)
    pay = row_payload(p, rows)
    t0 = time.perf_counter()
    done = vox = 0
    for k in range(0, rows.size, 20):
        n, v = row_work(prep[k:k + 20], pay[k:k + 20], consts)
        done += n
        vox += v
        if time.perf_counter() - t0 > budget_s:
            break
    t_rows = time.perf_counter() - t0
    per_refl = t_rows / max(done, 1) + t_prep * wl.n_frames / wl.n_refl
    return {"value": round(1.0 / per_refl, 2), "unit": UNIT, "cores": 1, "kind": "port",
            "voxels_per_s": round(vox / t_rows, 1),
            "sample": f"{done} reflections drawn at random from the workload (its mix of box shapes): gather, pass 1 "
                      f"and pass 2 by the numpy restatement in {t_rows:.1f} s, plus the full-frame preparation "
                      f"({t_prep * 1e3:.0f} ms per frame x {wl.n_frames} frames) shared over its {wl.n_refl} "
                      f"reflections"}


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
    D.keep_buffers(True)          # sweep after sweep: the pooled device buffers are kept between integrate() calls
    wl = Workload(args.workload, seed_offset=rank)
    src = wl.source()
    res = None
    for _ in range(args.warmup):  # results held across calls as in the timed loop: the pinned result buffers that
        res = wl.integrate(src)   # two live results need are allocated here, not in a timed step
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
        res = wl.integrate(src)
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
    t_max, n_total = reduce_over_ranks(t, wl.n_refl * args.steps, dist)
    value = n_total / t_max
    peak, peak_kind = _peaks()
    b_alg = alg_bytes(wl.spec, wl.n_frames, wl.plan) * args.steps * world
    pixel_gbs = b_alg / t_max / 1e9
    # roofline of the dominant kernel
    bpk = bytes_per_kernel(wl.plan, wl.n_frames)
    if "unpack" in ksum:
        bpk["unpack"] = 5.0 * wl.spec.nx * wl.spec.ny * wl.n_frames
    dom = max(ksum, key=lambda k: ksum[k][1]) if ksum else None
    roof = None
    if dom is not None:
        n_l, t_k = ksum[dom]
        per_launch = bpk.get(dom, 0.0) * args.steps / max(n_l, 1)
        achieved = per_launch / (t_k / n_l) / 1e9
        vox = float((wl.plan.Dz * wl.plan.bx.astype(np.float64) ** 2).sum()) * args.steps / max(n_l, 1)
        traffic = round(DRAM_BYTES_PER_VOXEL[dom] * vox / 1e9, 3) if dom in DRAM_BYTES_PER_VOXEL else None
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_unit": "GB per launch",
                "algorithmic": round(per_launch / 1e9, 3), "peak_kind": peak_kind,
                "launches": n_l, "ms_per_launch": round(t_k / n_l * 1e3, 4),
                "share": {k: round(v[1] / max(sum(x[1] for x in ksum.values()), 1e-12), 4) for k, v in ksum.items()},
                "ms_per_step": {k: round(v[1] / args.steps * 1e3, 2) for k, v in ksum.items()}}
    parity = None
    if rank == 0 and not args.no_parity:
        parity = _parity(wl, res_timed)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = _cpu_baseline(wl)
    # end to end: frames from pinned host memory, uploaded inside every step; results read back by the API
    e2e = None
    if not args.no_e2e:
        src = None                # the resident source holds the HBM copy of the packed frames
        wl.drop_resident()
        hsrc = wl.host_source()
        res = wl.integrate(hsrc)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        k2 = max(1, min(args.steps, args.e2e_steps))
        moved0 = dict(hsrc.transfer)
        f0.record()
        for _ in range(k2):
            res = wl.integrate(hsrc)
        f1.record()
        torch.cuda.synchronize()
        te, _ = reduce_over_ranks(f0.elapsed_time(f1) * 1e-3, 0, dist)
        n_out = sum(v.nbytes for v in res.refl.values() if isinstance(v, np.ndarray))
        moved = {k: (hsrc.transfer.get(k, 0) - moved0.get(k, 0)) / k2
                 for k in ("h2d_bytes", "chunks_raw", "chunks_packed")}
        e2e = {"value": round(wl.n_refl * world * k2 / te, 1), "unit": UNIT,
               "h2d_bytes_per_step": int(moved["h2d_bytes"]), "d2h_bytes_per_step": int(n_out), "steps": k2,
               "ms_per_step": round(te / k2 * 1e3, 1),
               "frames_on_host": ("packed transfer encoding, pinned" if wl.store is not None else "uint32, pinned"),
               "frame_bytes_per_step": int(4 * wl.spec.nx * wl.spec.ny * wl.n_frames)}
        if wl.store is None:
            e2e["chunks_per_step"] = {"raw": moved["chunks_raw"], "packed": moved["chunks_packed"]}
    if dist is not None:
        dist.barrier()
    if rank == 0:
        line = {"metric": METRICS[args.workload], "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(t_max / args.steps * 1e3, 3), "step_ms": step_ms,
                "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 accumulation)",
                "data": "synthetic: seeded 16M-pixel frames rendered on the device (spec in xpg_b200/synth.py)"
                        + ("; the sweep held in HBM in the packed transfer encoding (widened per wedge in the "
                           "timed region)" if wl.store is not None else ""),
                "config": workload_config(args.workload, wl.spec, wl.edges, wl.n_frames, wl.plan, world),
                "pixel_gbs": round(pixel_gbs, 1), "pixel_hbm_frac": round(pixel_gbs / peak, 4),
                "voxels_per_s": round(float((wl.plan.Dz * wl.plan.bx.astype(np.float64) ** 2).sum()) * args.steps
                                      * world / t_max, 1),
                "integrated_per_step": n_ok // max(args.steps, 1),
                "memory": {"block_parts": int(res_timed.memory["parts"]),
                           "open_buffers_gb": round(res_timed.memory["peak"] / 1e9, 1),
                           "budget_gb": round(res_timed.memory["budget"] / 1e9, 1)},
                "host_s_last_step": {k: round(v, 3) for k, v in res_timed.timing.get("host_s", {}).items()},
                "device_buffers": "kept between integrate() calls (xpg_b200.keep_buffers)",
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
                "parity": parity}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


_REF = {}


def _ref_init(consts):
    _REF["consts"] = consts


def _ref_worker(job):
    """Restatement work of one chunk of rows (prepared box frames, payloads) in a worker process."""
    prep, payload = job
    return row_work(prep, payload, _REF["consts"])


def _native_mapped():
    """Whether this process has mapped the library (it must not: the reference arm runs no code of this repo's
    library)."""
    try:
        return "libxpgi" in Path("/proc/self/maps").read_text()
    except OSError:
        return False


def reference_arm(args):
    """The reference's CPU path (its numpy restatement in oracle/) on all host cores, on the same workload and config
    as the device arm: the workload planned by the CPU restatement of the planner, then per step a uniform random
    sample of its reflections (gather, pass 1, pass 2 spread over spawned processes, from box windows of the same
    synthetic sweep rendered on the host) plus their share of the full-frame preparation XPG's frame loop does for
    every frame. No CUDA and none of this repository's library is used."""
    rank, world, local = _env()
    if rank != 0:
        return
    import multiprocessing as mp

    from oracle.pipeline import row_payload
    from oracle.plan import plan_integration
    from xpg_b200 import synth
    cores = len(os.sched_getaffinity(0))
    spec, exp, model, edges, n_frames, plan = plan_workload(args.workload, 0, plan_integration)
    _, table = synth.reflection_table(spec, z_range=(-5.0, n_frames + 5.0))

    def crop(f0, f1, y0, y1, x0, x1):
        return synth.render_window(spec, table, range(f0 + 1, f1 + 1), y0, y1, x0, x1)
    per_step = max(cores * 8, 96)
    n_all = per_step * 2                       # two distinct samples, cycled over the steps
    rows_all = random_rows(plan, n_all, seed=11)
    rng = np.random.default_rng(12)
    rows_all = rows_all[rng.permutation(rows_all.size)]
    prep_all = prepared_boxes(crop, plan, rows_all, n_frames, spec.ny, spec.nx, spec.overload)
    pay_all = row_payload(plan, rows_all)
    full = synth.render_window(spec, table, [1], 0, spec.ny, 0, spec.nx)
    t_prep = _frame_prep_seconds(full, spec.overload)
    consts = row_consts(spec, exp.geom, plan.nreg)
    ctx = mp.get_context("spawn")
    n_done, t_all, vox_all = 0, 0.0, 0
    with ctx.Pool(cores, initializer=_ref_init, initargs=(consts,)) as pool:
        def step(k):
            lo = (k * per_step) % max(rows_all.size - per_step + 1, 1)
            idx = list(range(lo, min(lo + per_step, rows_all.size)))
            jobs = [([prep_all[i] for i in idx[c::cores]], [pay_all[i] for i in idx[c::cores]]) for c in range(cores)]
            t0 = time.perf_counter()
            out = pool.map(_ref_worker, [j for j in jobs if j[1]])
            t_rows = time.perf_counter() - t0
            n = sum(o[0] for o in out)
            return n, sum(o[1] for o in out), t_rows + t_prep * n_frames / plan.n * n / cores
        for k in range(args.warmup):
            step(k)
        for k in range(args.steps):
            n, v, t = step(args.warmup + k)
            n_done += n
            vox_all += v
            t_all += t
    value = n_done / t_all
    line = {"metric": METRICS[args.workload], "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_all / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 accumulation)", "impl": "reference",
            "data": "synthetic: the same seeded sweep (spec in xpg_b200/synth.py), box windows rendered on the host",
            "config": workload_config(args.workload, spec, edges, n_frames, plan, world),
            "voxels_per_s": round(vox_all / t_all, 1),
            "cpu_baseline": {"value": round(value, 2), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{per_step} reflections per step drawn at random from the workload's "
                                       f"{plan.n} (its mix of box shapes): gather + pass 1 + pass 2 by the numpy "
                                       f"restatement over {cores} spawned processes, plus their share of the "
                                       f"full-frame preparation ({t_prep * 1e3:.0f} ms per frame x {n_frames} "
                                       f"frames over {cores} cores)"},
            "e2e": {"value": round(value, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "native_library_mapped": _native_mapped()}
    print(json.dumps(line), flush=True)


def _jobs_of(specs, wedge_frames, device="cuda"):
    """Batch jobs of synthetic sweeps whose frames are rendered on the device as the integration asks for them."""
    from xpg_b200 import synth
    from xpg_b200.batch import Job
    from xpg_b200.frames import GeneratedFrames
    from xpg_b200.plan import IntegrationModel
    jobs, n_refl = [], 0
    for s in specs:
        exp = s.experiment()
        _, table = synth.reflection_table(s, z_range=(-5.0, s.nframes + 5.0))
        spots = synth.DeviceSpots(s, table, device)
        edges = s.block_edges()
        jobs.append(Job(GeneratedFrames(spots, first=1, last=s.nframes, overload=s.overload, device=device),
                        [exp] * (len(edges) - 1), edges, IntegrationModel(sigma_d=s.sigma_d, sigma_m=s.sigma_m),
                        s.resolution_limit(), dict(frames=(1, s.nframes), n_regions_xy=s.n_regions_xy,
                                                   wedge_frames=wedge_frames), label=s.name))
    return jobs


def batched_bench(args):
    """Config 4: 12 sweeps (log-uniform 50..3600 frames, three detectors, three cells, sigma_M 0.05..0.5 deg),
    integrated one after another by `integrate()` (plain), together by the batched scheduler (shared persistent
    pass launches, admission by device footprint) and by the concurrent form (the plain path of several sweeps at
    once on host threads of their own); frames rendered on the device inside every timed region. One JSON line:
    reflections/s of each, the faster many-sweep form against plain, and that every result is the same bits."""
    import torch
    from xpg_b200 import device as D
    from xpg_b200 import synth
    from xpg_b200.batch import integrate_concurrent, run_jobs
    from xpg_b200.csrc import build
    from xpg_b200.integrate import integrate
    if build.stale():
        build.build()
    from xpg_b200 import memplan
    specs = synth.config4()
    jobs = _jobs_of(specs, WEDGE_FRAMES)
    budget = memplan.budget()          # one device budget for both forms: the same parts and passes, the same results

    def plain():
        return [integrate(j.images, j.exp_blocks, j.block_edges, j.model, j.dmin, verbose=False, mem_budget=budget,
                          **j.kwargs) for j in jobs]

    def batched():
        return run_jobs(jobs, budget_bytes=budget, bins=args.bins)

    def concurrent():
        return integrate_concurrent(jobs, budget_bytes=budget, workers=args.workers)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) * 1e-3
    for _ in range(max(args.warmup, 1)):
        timed(plain)
        timed(batched)
        timed(concurrent)
    tp, tb, tc, stats = [], [], [], None
    D.TIMER.reset()
    for _ in range(args.steps):
        rp, t = timed(plain)
        tp.append(t)
        (rb, stats), t = timed(batched)
        tb.append(t)
        (rc, cstats), t = timed(concurrent)
        tc.append(t)
    n = sum(len(r.refl["x"]) for r in rp)
    same = all(np.array_equal(a.refl[k], b.refl[k], equal_nan=True) for other in (rb, rc) for a, b in zip(rp, other)
               for k in ("isum", "iprf", "vprf", "bg", "isum_raw"))
    spans = {}
    if args.spans:                       # one more step of each, untimed, with device-time spans per kernel
        for name, fn in (("plain", plain), ("batched", batched)):
            D.TIMER.enabled = True
            D.TIMER.reset()
            _, t = timed(fn)
            torch.cuda.synchronize()
            spans[name] = {"seconds": round(t, 3), "device_s": {k: round(v[1], 4) for k, v in
                                                                D.TIMER.summary().items()}}
            D.TIMER.enabled = False
    rate = {"plain": n / np.median(tp), "batched": n / np.median(tb), "concurrent": n / np.median(tc)}
    best = max(("batched", "concurrent"), key=lambda k: rate[k])
    line = {"metric": "integrated reflections/s, 12 sweeps (config 4), batched vs plain", "unit": "refl/s",
            "value": round(rate[best], 1), "value_form": best, "plain": round(rate["plain"], 1),
            "batched_shared_launches": round(rate["batched"], 1), "concurrent": round(rate["concurrent"], 1),
            "speedup": round(rate[best] / rate["plain"], 3), "steps": args.steps, "warmup": args.warmup,
            "seconds": {"plain": [round(t, 3) for t in tp], "batched": [round(t, 3) for t in tb],
                        "concurrent": [round(t, 3) for t in tc]}, "workers": args.workers,
            "reflections": n, "same_results": bool(same),
            "sweeps": [{"frames": s.nframes, "detector": [s.nx, s.ny], "cell": s.space_group,
                        "sigma_m": round(s.sigma_m, 3), "reflections": len(r.refl["x"]),
                        "block_parts": int(r.memory["parts"]), "passes": len(r.memory.get("passes", [1])),
                        "planned_peak_gib": round(r.memory["peak"] / 2 ** 30, 1)} for s, r in zip(specs, rp)],
            "budget_gib": round(budget / 2 ** 30, 1), "spans": spans or None,
            "batched_stats": {k: (v if k != "host_s" else {a: round(b, 3) for a, b in v.items()})
                              for k, v in stats.items() if k in ("rounds", "blocks", "pass1_launches", "peak_bytes",
                                                                 "host_s")},
            "concurrent_stats": {"peak_bytes": cstats["peak_bytes"]},
            "data": "synthetic, frames rendered on the device inside the timed region (every form)"}
    print(json.dumps(line), flush=True)


def served_bench(args):
    """Config 5: concurrent sweeps of config 2's geometry (cells from config 4's list) whose 50-frame wedges arrive
    at 500 Hz per sweep with Poisson jitter (exponential gaps of 0.1 s mean between wedges); each arriving wedge is
    rendered on the device (the detector's frames landing in HBM) and fed to the request loop, which admits sweeps by
    device footprint and batches their completed blocks. One JSON line: p50 / p99 wedge-to-intensities latency
    against the 0.1 s acquisition time of a wedge, and sustained reflections/s."""
    import torch
    from xpg_b200 import synth
    from xpg_b200.batch import run_jobs
    from xpg_b200.csrc import build
    if build.stale():
        build.build()
    specs = synth.config5(nframes=args.served_frames, n_sweeps=args.served_sweeps)
    rng = np.random.default_rng(55)
    wedge = 50
    rate = float(args.served_rate)
    jobs = _jobs_of(specs, wedge)
    for j in jobs:
        nw = len(range(1, j.kwargs["frames"][1] + 1, wedge))
        j.arrivals = np.cumsum(rng.exponential(wedge / rate, nw))
    budget = args.served_budget_gb * 2 ** 30
    slots = len(jobs)
    warm = _jobs_of(specs[:1], wedge)
    warm[0].images.rereadable = False
    run_jobs(warm, budget_bytes=budget, bins=args.bins, slots=slots)    # warm-up: kernels loaded, allocator primed
    torch.cuda.synchronize()
    res, stats = run_jobs(jobs, budget_bytes=budget, bins=args.bins, served=True, slots=slots)
    lat = np.array([x[2] for x in stats["latency"]])
    comp = np.array([(x[0], x[1]) in stats["completing"] for x in stats["latency"]], bool)
    n = sum(len(r.refl["x"]) for r in res)
    last_arrival = max(float(j.arrivals[-1]) for j in jobs)

    def pct(v):
        return {"p50": round(float(np.percentile(v, 50)), 4), "p99": round(float(np.percentile(v, 99)), 4),
                "n": int(v.size)} if v.size else None
    line = {"metric": "served: wedge-to-intensities latency and sustained reflections/s (config 5)", "unit": "s",
            "p50": round(float(np.percentile(lat, 50)), 4), "p99": round(float(np.percentile(lat, 99)), 4),
            "max": round(float(lat.max()), 4), "wedge_acquisition_s": wedge / rate, "frame_rate_hz": rate,
            "sustained_refl_per_s": round(n / stats["seconds"], 1), "seconds": round(stats["seconds"], 3),
            "last_arrival_s": round(last_arrival, 3), "wedges": int(lat.size), "reflections": n,
            "latency_block_completing": pct(lat[comp]), "latency_other": pct(lat[~comp]),
            "budget_gib": args.served_budget_gb, "slots": slots,
            "sweeps": [{"frames": s.nframes, "cell": s.space_group, "reflections": len(r.refl["x"]),
                        "block_parts": int(r.memory["parts"]), "planned_peak_gib": round(r.memory["peak"] / 2 ** 30, 1)}
                       for s, r in zip(specs, res)],
            "scheduler": {k: (v if k != "host_s" else {a: round(b, 3) for a, b in v.items()})
                          for k, v in stats.items() if k in ("rounds", "blocks", "peak_bytes", "waits", "host_s")},
            "data": "synthetic; wedges rendered on the device at their arrival"}
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


def forward_bench(args):
    """The forward-model likelihood passes (xi_fm_scatter, xi_fm_gather; XPG's forward integrator on crowded data) on
    a window of 40 frames x a 1024 x 1024 tile holding 60,000 reflections of 9-frame, 13 x 13 px boxes with two
    separable terms (profile and halo), seeded factors; one step = one scatter (mu) and one gather of each mode, the
    passes of one Newton step of the intensity fit. One JSON line: voxel-terms per second and each pass's bandwidth
    against the HBM peak (algorithmic bytes: per box voxel, scatter 8 B of read-modify-write of mu; gather 6 B (int16
    counts, float32 mu) and, in mode 0, 4 B more; the factors once per reflection)."""
    import torch
    from xpg_b200 import forward as F
    from xpg_b200.csrc import build
    if build.stale():
        build.build()

    class Win:
        f0, f1, y0, ny, x0, nx = 0, 40, 0, 1024, 0, 1024
    n, T, Dz, b = 60000, 2, 9, 13
    g = torch.Generator(device="cuda").manual_seed(3)
    R = torch.rand((T, n, Dz), device="cuda", generator=g)
    P = torch.rand((T, n, b, b), device="cuda", generator=g) * 0.01
    iz0 = torch.randint(-4, 36, (n,), device="cuda", generator=g)
    iy0 = torch.randint(-6, 1018, (n,), device="cuda", generator=g)
    ix0 = torch.randint(-6, 1018, (n,), device="cuda", generator=g)
    rows = torch.arange(n, device="cuda")
    I = torch.rand(n, device="cuda", generator=g) * 100
    nv = 40 * 1024 * 1024
    M = torch.rand(nv, device="cuda", generator=g) + 0.1
    A = torch.rand(nv, device="cuda", generator=g)
    NS = torch.randint(-1, 8, (nv,), device="cuda", generator=g).to(torch.int16)
    mu = torch.zeros(nv, device="cuda")
    g0 = torch.zeros(n, device="cuda")
    g1 = torch.zeros(n, device="cuda")
    fd = torch.zeros(n, device="cuda")
    passes = {"scatter": lambda: F.scatter(mu, R, P, I, None, iz0, iy0, ix0, Win),
              "gather_ratio": lambda: F.gather(g0, None, R, P, rows, iz0, iy0, ix0, Win, A, M, NS, 0),
              "gather_newton": lambda: F.gather(g1, fd, R, P, rows, iz0, iy0, ix0, Win, None, M, NS, 1)}
    vox = n * Dz * b * b
    factors = n * T * (Dz + b * b) * 4
    alg = {"scatter": 8 * vox + factors, "gather_ratio": 10 * vox + factors, "gather_newton": 6 * vox + factors}
    peak, peak_kind = _peaks()
    out = {}
    for name, fn in passes.items():
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) * 1e-3 / args.steps
        out[name] = {"ms": round(t * 1e3, 3), "gbs": round(alg[name] / t / 1e9, 1),
                     "hbm_frac": round(alg[name] / t / 1e9 / peak, 4)}
    step = sum(v["ms"] for v in out.values()) * 1e-3
    line = {"metric": "forward-model likelihood passes: box voxel-terms per second (one scatter + two gathers)",
            "unit": "voxels/s", "value": round(3 * vox / step, 1), "steps": args.steps, "warmup": max(args.warmup, 3),
            "passes": out, "peak_gbs": peak, "peak_kind": peak_kind,
            "config": {"window": [40, 1024, 1024], "reflections": n, "box": [Dz, b, b], "terms": T},
            "data": "synthetic seeded factors, counts and model", "dtype": "f32 (per-reflection sums f64)"}
    print(json.dumps(line), flush=True)


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
    ap.add_argument("--workload", default="config2-sweep",
                    choices=("config2-sweep", "config2-block", "config2-small", "config1", "config4", "config5"))
    ap.add_argument("--bins", type=lambda v: tuple(int(x) for x in v.split(",")), default=None,
                    help="size bins (box sides) of the batched pass launches, e.g. 17,31,55,97")
    ap.add_argument("--served-frames", type=int, default=720, help="frames per sweep of the served workload")
    ap.add_argument("--served-rate", type=float, default=500.0, help="frames per second of each served sweep")
    ap.add_argument("--served-sweeps", type=int, default=4, help="concurrent sweeps of the served workload")
    ap.add_argument("--served-budget-gb", type=float, default=80.0,
                    help="device memory (GiB) the served sweeps are admitted under, one slot per sweep")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the post-check of the results against the oracle")
    ap.add_argument("--workers", type=int, default=3, help="config4: host threads of the concurrent form")
    ap.add_argument("--spans", action="store_true", help="config4: one more untimed step of each form with per-kernel "
                                                          "device-time spans")
    ap.add_argument("--decode", action="store_true", help="time the bitshuffle-LZ4 frame decode instead")
    ap.add_argument("--spots", action="store_true", help="time the spot-finding classifier instead")
    ap.add_argument("--forward", action="store_true", help="time the forward-model likelihood passes instead")
    args = ap.parse_args()
    if args.decode:
        decode_bench(args)
    elif args.forward:
        forward_bench(args)
    elif args.spots:
        spots_bench(args)
    elif args.workload == "config4" and args.impl != "reference":
        batched_bench(args)
    elif args.workload == "config5" and args.impl != "reference":
        served_bench(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
