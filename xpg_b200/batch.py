"""Batched and served integration: many sweeps on one GPU at once.

XPG integrates one sweep per call, one phi block after another, each shoebox shape and chunk of rows a separate
kernel call (`xpg/integrate.py:463-520`, the per-shape kernel cache `:347-351`). Here a scheduler keeps several sweeps'
integrations (`SweepRun`) open together:

* admission: a sweep starts when its device-memory footprint (the peak over its frames of the shoebox arenas and
  buffers of its open blocks, plus its wedge buffers; `footprint`) fits what the running sweeps leave of the budget,
  so sweeps that arrive while others run are admitted as memory frees up;
* each scheduler step feeds every running sweep its next wedge that has arrived (gathers into its open blocks);
* the blocks completed by a step, across sweeps, go through pass 1 together (one persistent launch per size bin of
  the box side, `xi_pass1_batched`), then each learns its profiles and widths, then pass 2 together
  (`xi_pass2_batched`), then results go to the host. Blocks of one sweep keep their order: a sweep contributes one
  block per round, so each block's pass 1 takes the widths adapted by the blocks before it.

Every result is the same number as the sweep integrated alone (`integrate`): the per-row arithmetic does not depend on
which rows share a launch, and each sweep's blocks are processed in its own order.

`integrate_batch` runs a list of sweeps as fast as possible (all frames available); `serve` replays requests whose
wedges arrive over time and reports the wedge-to-intensities latency of every wedge.
"""
from __future__ import annotations

import contextlib
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import device as D
from . import memplan
from .integrate import SweepRun


def block_bytes(plan, rows):
    """Device bytes a block holds while open (memplan.row_bytes of its rows)."""
    return int(memplan.row_bytes(plan)[rows].sum())


def footprint(plan, n_frames, wedge_bytes, depth=3):
    """Peak device bytes of a sweep's integration: the largest sum over its frames of the bytes of the blocks open
    at that frame (a block is open from the first frame any of its boxes needs to its last), plus `depth` wedge
    buffers. The device counterpart of XPG's host-memory pass planning (`_plan_passes`, xpg/shoebox.py:134-196),
    which sizes the same open-block curve against host memory."""
    d = np.zeros(n_frames + 2, np.float64)
    for b, rows in enumerate(plan.blocks_refl):
        if rows.size:
            lo = int(np.clip(plan.need_lo[b], 0, n_frames))
            hi = int(np.clip(plan.need_hi[b] + 1, 0, n_frames + 1))
            w = block_bytes(plan, rows)
            d[lo] += w
            d[hi] -= w
    return int(np.cumsum(d).max()) + depth * wedge_bytes


def job_footprint(job, device="cuda"):
    """Device bytes a job needs when it runs (planned here; nothing is integrated)."""
    run = SweepRun(job.images, job.exp_blocks, job.block_edges, job.model, job.dmin, early_pass1=False,
                   device=device, verbose=False, mem_budget=float("inf"), **job.kwargs)
    try:
        wb = max(fb - fa + 1 for fa, fb in run.wedges) * run.src.ny * run.src.nx * 4
        return footprint(run.plan, run.wedges[-1][1], wb)
    finally:
        run.close()


@dataclass
class Job:
    """One sweep to integrate: `integrate()`'s arguments (images: a frame source), an optional label, and for
    serving the arrival time of each of its wedges (seconds after the request loop starts)."""
    images: object
    exp_blocks: list
    block_edges: np.ndarray
    model: object
    dmin: float
    kwargs: dict = field(default_factory=dict)
    arrivals: np.ndarray | None = None
    label: str = ""


class _Active:
    def __init__(self, i, job, run, nbytes):
        self.i, self.job, self.run, self.nbytes = i, job, run, nbytes
        self.w = 0                         # next wedge to feed
        self.pend = []                     # completed blocks waiting for processing, in processing order
        self.t_start = None


def _round(active, bins, stats):
    """One batched round: the first pending block of every sweep with one, through pass 1, learning, pass 2 and
    collection. Returns the (sweep, block) pairs processed."""
    picks = [(a, a.pend.pop(0)) for a in active if a.pend]
    if not picks:
        return []
    sets1, groups = [], []
    for k, (a, b) in enumerate(picks):
        e, rem = a.run.pass1_stage(b, batched=True)
        rs = a.run.live[b].rowset
        sets1.append(e)
        groups.append((k, rem, rs.bx[rem], rs.Dz[rem]))
    dev = active[0].run.device
    if any(len(g[1]) for g in groups):
        t1 = D.RowSetTable(sets1, dev)
        D.pass1_batched(t1, D.batched_items(groups, bins, dev))
        stats["pass1_launches"] += 1
    for a, b in picks:
        a.run.learn(b)
    sets2, groups2 = [], []
    for a, b in picks:
        e = a.run.pass2_stage(b, batched=True)
        if e is not None:
            rs = a.run.live[b].rowset
            groups2.append((len(sets2), np.arange(rs.n), rs.bx, rs.Dz))
            sets2.append(e)
    if sets2:
        t2 = D.RowSetTable(sets2, dev)
        D.pass2_batched(t2, D.batched_items(groups2, bins, dev))
    for a, b in picks:
        a.run.collect(b)
    stats["rounds"] += 1
    stats["blocks"] += len(picks)
    return picks


def run_jobs(jobs, budget_bytes=None, bins=None, device="cuda", served=False, clock=time.perf_counter,
             on_wedge=None, max_active=None, graphs=False, slots=None, overlap=True):
    """Integrates `jobs` (list of Job) together; returns (results in job order, stats). served: each wedge is fed no
    earlier than its arrival time (job.arrivals, seconds after the start) and the latency of every wedge (from its
    arrival to the completion of everything it triggered: its gathers and, when it completes blocks, their
    intensities on the host) is recorded in stats["latency"]. graphs: each sweep's per-wedge gathers replayed from
    a CUDA graph (captured once per set of open blocks). overlap: each sweep's gathers on a stream of its own, beside
    the passes of every sweep's completed blocks. slots: each sweep is planned (blocks in parts, memplan.fit)
    for budget_bytes / slots, so that `slots` sweeps run at once; by default each is planned for the whole budget
    and sweeps wait for the memory the running ones hold."""
    budget = budget_bytes if budget_bytes is not None else int(0.8 * torch.cuda.mem_get_info(device)[0])
    plan_budget = budget / slots if slots else budget
    queue = list(range(len(jobs)))
    active, results = [], [None] * len(jobs)
    used = 0
    stats = dict(rounds=0, blocks=0, pass1_launches=0, latency=[], admitted_at={}, peak_bytes=0, waits=0,
                 completing=set(), host_s=dict(feed=0.0, rounds=0.0, admit=0.0, finish=0.0))
    hs = stats["host_s"]
    t0 = clock()

    def arrived(a, w):
        if not served or a.job.arrivals is None:
            return True
        return clock() - t0 >= a.job.arrivals[w]

    head = {}                                                # the planned run at the head of the queue

    def admit():
        nonlocal used
        while queue and (max_active is None or len(active) < max_active):
            i = queue[0]
            job = jobs[i]
            if served and job.arrivals is not None and clock() - t0 < job.arrivals[0]:
                return                                       # the request has not arrived
            if i not in head:
                if served:
                    job.images.rereadable = False            # live frames arrive once: no second pass over them
                run = SweepRun(job.images, job.exp_blocks, job.block_edges, job.model, job.dmin, early_pass1=False,
                               device=device, verbose=False, mem_budget=plan_budget, graphs=graphs,
                               overlap=overlap, **job.kwargs)
                head[i] = (run, int(run.mem["peak"]))              # parts and passes included
            run, need = head[i]
            if active and used + need > budget:
                return                                       # waits for memory to free up
            del head[i]
            used += need
            queue.pop(0)
            a = _Active(i, job, run, need)
            a.t_start = clock() - t0
            stats["admitted_at"][i] = a.t_start
            active.append(a)
            stats["peak_bytes"] = max(stats["peak_bytes"], used)

    waiting = []                                             # (job, wedge, event, arrival) of fed wedges
    admit()
    while active or queue or waiting:
        progressed = False
        fed = []
        for a in active:
            if a.w < len(a.run.wedges) and arrived(a, a.w):
                t_ = time.perf_counter()
                got = a.run.feed(a.w)
                hs["feed"] += time.perf_counter() - t_
                if got:
                    stats["completing"].add((a.i, a.w))     # the wedge completed blocks: its latency has their passes
                a.pend += got
                fed.append((a, a.w))
                a.w += 1
                progressed = True
            if a.w >= len(a.run.wedges) and not a.pend and a.run.opened:
                a.pend += a.run.remaining()
            if (a.w >= len(a.run.wedges) and not a.pend and not a.run.opened and not a.run.live
                    and a.run.pass_index + 1 < a.run.n_passes):
                a.run.start_pass(a.run.pass_index + 1)       # blocks that did not fit in one pass over the frames
                a.w = 0
                progressed = True
        t_ = time.perf_counter()
        while any(a.pend for a in active):
            _round(active, bins, stats)
            progressed = True
        hs["rounds"] += time.perf_counter() - t_
        if served and fed:
            # a wedge is done when the work queued for it (its gathers, and the blocks it completed, whose results
            # are on the host already) has run: an event after it, polled without stopping the loop
            for a, w in fed:
                ev = torch.cuda.Event()
                ev.record()
                evs = (ev,) if a.run.last_gathered is None else (ev, a.run.last_gathered)
                waiting.append((a.i, w, evs, float(a.job.arrivals[w]) if a.job.arrivals is not None else 0.0))
        if waiting:
            now = clock() - t0
            left = []
            for i, w, ev, arr in waiting:
                if all(e.query() for e in ev):
                    stats["latency"].append((i, w, now - arr))
                    if on_wedge is not None:
                        on_wedge(i, w, now)
                else:
                    left.append((i, w, ev, arr))
            waiting[:] = left
        for a in [a for a in active if a.w >= len(a.run.wedges) and not a.pend and not a.run.opened
                  and a.run.pass_index + 1 >= a.run.n_passes]:
            t_ = time.perf_counter()
            results[a.i] = a.run.result()
            hs["finish"] += time.perf_counter() - t_
            a.run.close()
            used -= a.nbytes
            active.remove(a)
            progressed = True
        n_before = len(active)
        t_ = time.perf_counter()
        admit()
        hs["admit"] += time.perf_counter() - t_
        progressed = progressed or len(active) != n_before
        if not progressed:
            stats["waits"] += 1
            time.sleep(2e-4)                                 # nothing has arrived yet
    stats["seconds"] = clock() - t0
    return results, stats


@contextlib.contextmanager
def _own_stream(device):
    """The calling thread's device work on a CUDA stream of its own (made current), waited for on exit."""
    dev = torch.device(device)
    with torch.cuda.device(dev if dev.index is not None else torch.cuda.current_device()):
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            yield stream
        stream.synchronize()


def integrate_concurrent(jobs, budget_bytes=None, workers=3, device="cuda"):
    """Integrates every job (all frames available) on `workers` host threads, each running the plain path of one
    sweep at a time (`integrate.drive`) on streams of its own: one sweep's host stages (planning, adaptation,
    result assembly) and waits for its own device work overlap the other sweeps' device work. Each sweep is planned
    for the whole budget, exactly as `integrate(..., mem_budget=budget_bytes)` plans it, and starts once its planned
    peak fits beside the running sweeps' (the largest runs alone), so every result is the same bits as the sweep
    integrated alone under that budget. Returns (results in job order, stats)."""
    import threading
    from concurrent.futures import ThreadPoolExecutor

    from .integrate import drive
    budget = budget_bytes if budget_bytes is not None else memplan.budget(device)
    cond = threading.Condition()
    state = dict(used=0, running=0, peak=0)
    results = [None] * len(jobs)
    t0 = time.perf_counter()
    stats = dict(admitted_at={}, peak_bytes=0, workers=workers)

    def work(i):
        job = jobs[i]
        with _own_stream(device):
            run = SweepRun(job.images, job.exp_blocks, job.block_edges, job.model, job.dmin, verbose=False,
                           device=device, mem_budget=budget, overlap=True, **job.kwargs)
            need = int(run.mem["peak"])
            try:
                with cond:
                    while state["running"] and state["used"] + need > budget:
                        cond.wait()
                    state["used"] += need
                    state["running"] += 1
                    stats["peak_bytes"] = max(stats["peak_bytes"], state["used"])
                    stats["admitted_at"][i] = time.perf_counter() - t0
                try:
                    results[i] = drive(run)
                finally:
                    with cond:
                        state["used"] -= need
                        state["running"] -= 1
                        cond.notify_all()
            finally:
                run.close()

    with ThreadPoolExecutor(max_workers=max(int(workers), 1)) as ex:
        for f in [ex.submit(work, i) for i in range(len(jobs))]:
            f.result()
    stats["seconds"] = time.perf_counter() - t0
    return results, stats


def integrate_batch(jobs, budget_bytes=None, bins=None, device="cuda"):
    """Integrates every job (all frames available) with batched rounds; results in job order."""
    res, stats = run_jobs(jobs, budget_bytes, bins, device)
    return res


def serve(jobs, budget_bytes=None, bins=None, device="cuda", slots=None):
    """Request loop over jobs whose wedges arrive at job.arrivals: (results, stats) with the per-wedge latency.
    slots: sweeps planned to run at once within budget_bytes (run_jobs)."""
    return run_jobs(jobs, budget_bytes, bins, device, served=True, slots=slots)
