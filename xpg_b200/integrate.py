"""Drop-in for XPG's integration stage (`xpg/integrate.py`): `integrate`, `estimate_sigmas`, `IntegrationModel`,
`IntegrationResult` with the reference's signatures (`:197-215`, `:1002-1003`), computed on one B200.

Data flow of a sweep:
  host   predictions and the shoebox plan (xpg_b200.plan), block by block;
  device frames arrive in wedges of consecutive frames (uploaded from host memory, or already resident); one
         launch per (open block, wedge) gathers every box window into the block's shoebox arena (value + 3,
         binned rows as IEEE-encoded sums);
  device when a block's last frame has arrived: bin decode, pass 1, strong-row profile accumulation (float64
         grids), profile finalisation, pass 2; the host adapts sigma_M / rocking curve / sigma_D in between
         (float64, xpg_b200.adapt) from the block's strong rows.
Blocks are processed in the order they complete, so the adaptive widths carry over exactly as in the reference.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import adapt as A
from . import device as D
from . import memplan
from . import native as N
from .frames import as_frame_source
from .geometry import centring_allowed
from .plan import DZ_BUCKETS, IntegrationModel, plan_integration

PROFILE_GRID = 41
MAX_DZ = max(DZ_BUCKETS)
WEDGE_FRAMES = 32                     # frames per upload / gather launch
EARLY_PASS1_ROWS = 16384              # completed rows worth an early pass-1 launch (uploaded frames)
LOOKAHEAD = 2                         # wedges gathered (overlap mode) before the passes of a block they completed
OUT_F64 = ("bg", "isum", "vsum", "vsum0", "iprf", "vprf", "vprf0", "corr", "xo", "yo", "zo", "p_valid", "p_total",
           "frac_rec", "rho", "m_d", "m_m", "p_fg")


@dataclass
class IntegrationResult:
    refl: dict
    model: IntegrationModel
    profiles: dict = field(default_factory=dict)
    timing: dict = field(default_factory=dict)


class _Block:
    """Device state of one phi block: its row tables and schedule (made ahead, while the host waits for the device),
    then its shoebox arena (`allocate`, when the block opens)."""

    def __init__(self, b, rows, plan, device):
        self.b = b
        self.rows = rows                                  # global row indices, reference kernel-call order
        p = plan
        dv = p.dev                                        # the planner's device columns
        if rows.size and rows[-1] - rows[0] + 1 == rows.size and (rows[1:] > rows[:-1]).all():
            a, e = int(rows[0]), int(rows[-1]) + 1        # a range of plan rows (the planner's block order): views
            sel = lambda t: t[a:e]
        else:
            rt = D.h2d(rows, None, device)
            sel = lambda t: t.index_select(0, rt)
        pj = sel(dv["nbj"][:, 0]).long()                  # nearest neighbour: the partner where there is one
        rad = lambda phi: (phi * (np.pi / 180.0)).float()  # numpy's radians, then float32
        nb = {k: sel(dv["nb" + k]) for k in ("x", "y", "z", "sx", "sz")}
        if nb["x"].shape[1] != p.nb_columns:              # foreign-spot columns were added on the host
            nb = {k: v[rows] for k, v in p.nb.items()}
        ix0, iy0, iz0, fb, pxs = (sel(dv[k]) for k in ("ix0", "iy0", "iz0", "fb", "pxs"))
        self.rowset = D.RowSet(
            S=sel(dv["S"]).float(), phi=rad(sel(dv["phi"])), ix0=ix0, iy0=iy0, iz0=iz0, fb=fb,
            region=sel(dv["region"]), has_p=sel(dv["has_partner"]), pS=dv["S"].index_select(0, pj).float(),
            pphi=rad(dv["phi"].index_select(0, pj)), pxs=pxs, Dz=p.Dz[rows], bx=p.bx[rows], nb=nb, device=device,
            sb_bias=3.0)
        self.grows = D.GatherRows(self.rowset, ix0, iy0, iz0, p.fb[rows], pxs, device)
        self.arena = None
        self.cnt = None
        ident = bool((rows[1:] > rows[:-1]).all())         # local rows by global row: outputs leave in plan order
        order = None if ident else np.argsort(rows, kind="stable")
        self.perm_t = None if ident else D.h2d(order, None, device)
        self.rows_sorted = rows if ident else rows[order]
        srt = self.rows_sorted
        self.span = (int(srt[0]), int(srt[-1]) + 1) if srt.size and srt[-1] - srt[0] + 1 == srt.size else None
        self.z_lo = p.iz0[rows].astype(np.int64)
        self.z_hi = self.z_lo + self.grows.span - 1      # last frame index a row's box can take
        self.comp_hi = self.z_hi                          # last frame a row receives (set by schedule())
        self.p1 = None                                    # pass-1 buffers and constants, made at the first pass 1
        self.c1 = None
        self.p1_done = np.zeros(rows.size, bool)
        # gather order: rows by 128-pixel detector tile (row-major), plan order within a tile, so that the boxes the
        # resident CTAs gather at one time overlap on the detector and share their frame pixels in L2
        pxs_h = p.pxs[rows].astype(np.int64)
        tile = ((p.iy0[rows] * pxs_h) // 128 + 64) * 4096 + (p.ix0[rows] * pxs_h) // 128 + 64
        self.by_tile = np.argsort(tile, kind="stable").astype(np.int32)
        self.z_lo_t, self.z_hi_t = self.z_lo[self.by_tile], self.z_hi[self.by_tile]

    def allocate(self, device, f_lo, eff_hi, zero_all):
        """The shoebox arena (from the buffer pool) and bin counters: the block opens. A slot must read 0 wherever no
        frame is gathered into it. The block gathers every frame from f_lo (the first frame index of the run) or
        its first row's, up to eff_hi (its last gathered frame), so the gathers write the whole slot of a plain row
        whose box frames (all Dz of them, the depth bucket's padding included) lie in [f_lo, eff_hi]; only the
        others are cleared: binned rows (they accumulate), rows starting before the run, rows whose padded depth
        reaches past eff_hi, or every row when frames are excluded."""
        self.arena = D.POOL.take(max(self.rowset.n_vox, 1), torch.float32, device)
        need = self.grows.binned | (self.z_lo < f_lo) | (self.z_hi > eff_hi)
        if zero_all or need.all():
            self.arena.zero_()
        elif need.any():
            D.zero_rows(self.grows, self.arena, D.h2d(np.flatnonzero(need).astype(np.int32), None, device))
        self.cnt = torch.zeros(max(self.grows.n_cnt, 1), dtype=torch.int32, device=device)

    def rows_in(self, fi_a, fi_b):
        """Local rows whose box frame range meets [fi_a, fi_b]."""
        return np.flatnonzero((self.z_lo <= fi_b) & (self.z_hi >= fi_a)).astype(np.int32)

    def schedule(self, wedges, eff_hi, early_rows, device):
        """The block's per-wedge index lists, computed at block open and uploaded in one copy: the rows each wedge
        gathers into, and (early_rows > 0) the launch groups of the rows whose last frame arrives with a wedge, batched
        to at least early_rows rows. One upload before the frame transfers: a small copy issued later would wait in
        the copy engine behind every frame wedge already queued."""
        self.comp_hi = np.minimum(self.z_hi, eff_hi)
        parts, off = [], 0

        def add(a):
            nonlocal off
            parts.append(np.asarray(a, np.int32))
            o = off
            off += parts[-1].size
            return o, parts[-1].size
        self.w_gather, self.w_early = {}, {}
        acc = np.zeros(0, np.int64)
        first = int(self.z_lo.min()) if self.z_lo.size else 0
        for w, (fa, fb) in enumerate(wedges):
            fi_a, fi_b = fa - 1, fb - 1
            if fi_b < first or fi_a > eff_hi:              # wedges before or after the block's frames
                continue
            if eff_hi >= fi_a:
                hi = min(fi_b, eff_hi)
                loc = self.by_tile[(self.z_lo_t <= hi) & (self.z_hi_t >= fi_a)]     # in gather (tile) order
                if loc.size:
                    self.w_gather[w] = add(loc)
            if early_rows:
                acc = np.concatenate([acc, np.flatnonzero((self.comp_hi <= fi_b) & (self.comp_hi >= fi_a))])
                if acc.size >= early_rows:
                    groups = [(bx, dz, add(o)) for bx, dz, o in D.host_groups(self.rowset, acc)]
                    binned = acc[self.grows.binned[acc]]
                    self.w_early[w] = (acc, groups, add(binned) if binned.size else None)
                    acc = np.zeros(0, np.int64)
        self.sched_t = D.h2d(np.concatenate(parts) if parts else np.zeros(1, np.int32), None, device)

    def sched(self, o_n):
        o, n = o_n
        return self.sched_t[o:o + n]


def integrate(images, exp_blocks, block_edges, model: IntegrationModel, dmin, dmax=1e9, frames=None, mask=None,
              minimum_zeta=0.05, verbose=True, log=print, n_regions_xy=3, learn_profiles=True, exclude_frames=(),
              adaptive=True, deconvolve_overlaps=True, extra_lattices=None, bkg_template=None, foreign_spots=None,
              n_foreign=4, moments_only=False, *, wedge_frames=WEDGE_FRAMES, device="cuda", allowed=centring_allowed,
              graphs=False, mem_budget=None, overlap=True):
    """Integrate a sweep (`xpg/integrate.py:209-999`). `exp_blocks`: one experiment per phi block, `block_edges` in
    frame-coordinate units; `extra_lattices`: further lattices integrated together (refl['lattice'] = id); graphs:
    each wedge's gathers replayed from a CUDA graph captured once per set of open blocks; mem_budget: device bytes the
    open blocks' buffers may use (default: memplan.budget), beyond which blocks are integrated in parts; overlap (on
    by default; results are the same bits either way): the gathers on a stream of their own, LOOKAHEAD wedges ahead
    of the passes of the blocks they completed."""
    run = SweepRun(images, exp_blocks, block_edges, model, dmin, dmax, frames, mask, minimum_zeta, verbose, log,
                   n_regions_xy, learn_profiles, exclude_frames, adaptive, deconvolve_overlaps, extra_lattices,
                   bkg_template, foreign_spots, n_foreign, moments_only, wedge_frames=wedge_frames, device=device,
                   allowed=allowed, graphs=graphs, mem_budget=mem_budget, overlap=overlap)
    try:
        return drive(run)
    finally:
        run.close()


def drive(run):
    """Runs a planned sweep (`SweepRun`) through its frame loop and returns its result: wedges fed in order, each
    completed block processed once the gathers of LOOKAHEAD later wedges are queued (overlap mode), then the blocks
    left open, then further passes over the frames when the memory plan asks for them."""
    ahead = LOOKAHEAD if run.gs is not None else 0
    done = []                                        # (block, wedge that completed it), in processing order
    for w in range(len(run.wedges)):
        done += [(b, w) for b in run.feed(w)]
        while done and w - done[0][1] >= ahead:      # later wedges' gathers are queued before a block's passes
            run.process(done.pop(0)[0])
        run.early_pass1(w)
    for b, _ in done:
        run.process(b)
    for b in run.remaining():
        run.process(b)
    for k in range(1, run.n_passes):                 # blocks that did not fit in one pass over the frames
        run.start_pass(k)
        for w in range(len(run.wedges)):
            for b in run.feed(w):
                run.process(b)
        for b in run.remaining():
            run.process(b)
    return run.result()


class SweepRun:
    """One sweep's integration as a sequence of stages a scheduler can interleave with other sweeps': `feed(w)`
    gathers wedge w into the open blocks and returns the blocks it completed (in the order they are processed); a
    completed block then goes through `pass1_stage` (bin decode; pass 1 of its rows not done yet, or their launch
    items for a batched launch), `learn` (profile accumulation, the adaptation of the widths on the host, profile
    finalisation, pass-2 constants), `pass2_stage` (pass 2, or its items) and `collect` (results to the host).
    `process(b)` runs the four in order. Blocks of one sweep must be processed in the order feed / remaining return
    them: each block's pass 1 takes the widths adapted by the blocks processed before it."""

    def __init__(self, images, exp_blocks, block_edges, model, dmin, dmax=1e9, frames=None, mask=None,
                 minimum_zeta=0.05, verbose=True, log=print, n_regions_xy=3, learn_profiles=True, exclude_frames=(),
                 adaptive=True, deconvolve_overlaps=True, extra_lattices=None, bkg_template=None, foreign_spots=None,
                 n_foreign=4, moments_only=False, *, wedge_frames=WEDGE_FRAMES, device="cuda",
                 allowed=centring_allowed, early_pass1=True, plan=None, mem_budget=None, graphs=False,
                 overlap=False):
        N.require_cuda()
        self.t0 = time.time()
        lattice_of = [0] * len(exp_blocks)
        if extra_lattices:
            exp_blocks = list(exp_blocks)
            for li, lat in enumerate(extra_lattices, start=1):
                exp_blocks += list(lat)
                lattice_of += [li] * len(lat)
        self.exp_blocks = exp_blocks
        src = as_frame_source(images, device)
        if frames is None:
            frames = (src.first, src.last)
        f_first, f_last = int(frames[0]), int(frames[1])
        excl = set(int(f) for f in exclude_frames)
        # wedges of the run; frames in pinned host memory start moving to the device now, under the planning
        self.resident = resident = bool(getattr(src, "resident", False))
        W = (f_last - f_first + 1) if resident else max(int(wedge_frames), 1)    # resident: one wedge, one gather
        self.wedges = [(f, min(f + W - 1, f_last)) for f in range(f_first, f_last + 1, max(W, 1))]
        self.oks = [np.array([(g_ not in excl) for g_ in range(fa, fb + 1)], bool) for fa, fb in self.wedges]
        self.f_range = (f_first - 1, f_last - 1)              # frame indices the run integrates
        self.any_excluded = not all(ok.all() for ok in self.oks)
        self.src = src
        self.feeder = src.feeder(self.wedges, self.oks) if (hasattr(src, "feeder") and not resident) else None
        self.device, self.model, self.verbose, self.log = device, model, verbose, log
        self.learn_profiles, self.adaptive, self.moments_only = learn_profiles, adaptive, moments_only
        self.plan = p = plan if plan is not None else plan_integration(
            exp_blocks, block_edges, model, dmin, dmax, (f_first, f_last), minimum_zeta, n_regions_xy, adaptive,
            deconvolve_overlaps, lattice_of, foreign_spots, n_foreign, allowed)
        # device memory: blocks split into parts of consecutive phi when their open buffers exceed the budget
        wedge_bytes = 0 if resident else 3 * W * src.ny * src.nx * 4
        limit = mem_budget if mem_budget is not None else memplan.budget(device)
        self.plan, exp_blocks, self.mem = memplan.fit(p, exp_blocks, f_last, wedge_bytes, limit,
                                                      allow_passes=getattr(src, "rereadable", True))
        p = self.plan
        self.exp_blocks = exp_blocks
        self.refl = p.refl
        n = p.n
        if D.POOL.persist and D.POOL.free:    # buffers kept from the last run: only those this run's blocks can take
            b2 = p.bx.astype(np.int64) ** 2
            vox_row = b2 * p.Dz
            vox = [int(memplan._rows_sum(vox_row, r)) for r in p.blocks_refl]
            pix = [17 * int(memplan._rows_sum(b2, r)) for r in p.blocks_refl]
            D.POOL.retain({torch.float32: vox, torch.uint8: pix, torch.int32: [W * src.ny * src.nx]})
        if verbose and (self.mem["parts"] > 1 or "passes" in self.mem):
            log(f"  INTEGRATE: open shoebox buffers ~{self.mem['one'] / 2 ** 30:.1f} GB > the device budget "
                f"{limit / 2 ** 30:.1f} GB: each phi block in {self.mem['parts']} parts, "
                f"{len(self.mem.get('passes', [1]))} passes over the frames, peak ~{self.mem['peak'] / 2 ** 30:.1f} GB")
        if verbose:
            log(f"  INTEGRATE: {p.info['n_predicted']} predicted reflections, box {p.box}x{p.box} px, sigma_D "
                f"{model.sigma_d:.4f} sigma_M {model.sigma_m:.4f} deg; {p.info['n_wide']} wide in phi (> {MAX_DZ} "
                f"frames): integrated in bins, {p.info['n_trunc']} of them still truncated")
        self.out = out = {k: np.empty(n, np.float64) for k in OUT_F64}     # every processed block fills its rows
        out["n_over"] = np.zeros(n, np.int32)
        out["n_fg_masked"] = np.zeros(n, np.int32)
        out["isum_raw"] = np.full(n, -1, np.int64)                 # -1: not integrated (rows of no processed block)
        self.fz_out = np.zeros((n, MAX_DZ), np.float32) if not learn_profiles else None
        self.nreg = p.nreg
        self.sd = np.radians(model.sigma_d)
        self.sm = np.radians(model.sigma_m)
        self.state = dict(sd=self.sd, sm=self.sm, rcw=A.rc_default_weights())
        self.block_params, self.prof_by_block, self.block_widths = {}, {}, {}
        self.t_dev = 0.0
        self.host_s = {"plan": time.time() - self.t0}     # host seconds per stage (waits for the device included)
        nblocks = len(exp_blocks)
        self.read_fi = read_fi = np.array([f - 1 for f in range(f_first, f_last + 1) if f not in excl], np.int64)
        # a block takes every frame read up to the first frame read at or after its last needed frame
        # (`xpg/integrate.py:789-793`: completion is checked after the frame's gather)
        self.eff_hi = {}
        for b in range(nblocks):
            if p.blocks_refl[b].size:
                k = np.searchsorted(read_fi, p.need_hi[b], "left")
                self.eff_hi[b] = int(read_fi[min(k, len(read_fi) - 1)]) if len(read_fi) else -1
        # passes over the frames (memplan, when the open blocks do not fit even in parts): each reads every frame
        self.passes = self.mem.get("passes") or [[b for b in range(nblocks) if p.blocks_refl[b].size]]
        self.n_passes = len(self.passes)
        self.pass_index = 0
        self.pending = sorted(self.passes[0], key=lambda b: p.need_lo[b])
        self.opened, self.open_order = {}, []
        self.prepared = {}                # blocks made ahead of their opening (prepare_ahead)
        self.det_cache = {}
        self.bkg_template = bkg_template
        self.mask_t = None
        if mask is not None and not np.asarray(mask).all():
            self.mask_t = D.h2d(np.asarray(mask, np.uint8), None, device)
        self.processed = []
        self.collects = []                # blocks whose results are on their way to the host (collect -> finish)
        self.live = {}                    # completed blocks between pass1_stage and collect
        # when frames are uploaded, rows of the next block to complete whose last frame has arrived get their pass 1
        # as soon as their wedge is in: it overlaps the transfer of the later wedges (their widths are fixed: every
        # block before it has been processed). Resident frames have no transfer to hide: their blocks run pass 1
        # whole, in the fewest launches.
        ok_parts = [ok.astype(np.uint8) for ok in self.oks if not ok.all()]
        self.ok_dev = D.h2d(np.concatenate(ok_parts), None, device) if ok_parts else None
        self.ok_off = 0
        # (sources whose frames are produced in HBM have no transfer to hide)
        hide = bool(getattr(src, "hide_transfer", True))
        self.early_rows = EARLY_PASS1_ROWS if (early_pass1 and not resident and hide) else 0
        self.graphs = graphs and not resident     # per-wedge gathers replayed from a CUDA graph (GatherGraph)
        self._gg = None
        self.reported = set()                     # completed blocks handed out by feed / remaining
        # overlap: gathers on a stream of their own, so that they run beside the passes and the host's work on
        # completed blocks (which then wait for their blocks' gathers only); blocks' pass-1 widths are taken when
        # their pass 1 runs, so early pass 1 (which takes them at block opening) is off
        self.gs = torch.cuda.Stream(device=device) if (overlap and not resident) else None
        self.last_gathered = None
        if self.gs is not None:
            self.early_rows = 0

    # ---- device constants
    def detector(self, g):
        key = (id(g), id(self.bkg_template))
        if key not in self.det_cache:
            self.det_cache.clear()
            self.det_cache[key] = D.DeviceDetector(g, self.bkg_template, self.device)
        return self.det_cache[key]

    def widths(self):
        st = self.state
        sd_b = st["sd"] if self.adaptive else self.sd
        sm_b, rcw_b = (st["sm"], st["rcw"]) if self.adaptive else (self.sm, A.rc_default_weights())
        return sd_b, sm_b, rcw_b

    def _prepare(self, b):
        blk = _Block(b, self.plan.blocks_refl[b], self.plan, self.device)
        blk.schedule(self.wedges, self.eff_hi[b], self.early_rows, self.device)
        return blk

    def prepare_ahead(self, n=1):
        """Row tables and schedules of the next n blocks to open, made while the host would otherwise wait for the
        device (their opening then only takes the arena)."""
        t0 = time.perf_counter()
        for b in self.pending[:n]:
            if b not in self.prepared:
                self.prepared[b] = self._prepare(b)
        self._clock("prepare", t0)

    def block_pass1_consts(self, b, blk: _Block):
        """The block's pass-1 constants from the current widths (those adapted by every block processed before it),
        made once; allocated with the buffers before any frame transfer of the block is queued."""
        if blk.p1 is None:
            sd_b, sm_b, rcw_b = self.widths()
            blk.c1 = (sd_b, sm_b, rcw_b) + D.block_consts(self.exp_blocks[b].geom, sd_b, sm_b, self.model.gain,
                                                          rcw_b, self.device)
            blk.p1 = D.Pass1Buffers(blk.rowset, pooled=True)

    def pass1_rows(self, b, blk: _Block, idx, groups=None, binned_t=None):
        """Bin decode and pass 1 of the block's local rows idx, whose frames have all been gathered (launch groups
        and binned rows on the device when given, else made here)."""
        self.decode_rows(b, blk, idx, binned_t)
        if groups is None and idx.size != blk.rowset.n:
            groups = D.subset_groups(blk.rowset, idx)
        D.pass1(self.detector(self.exp_blocks[b].geom), blk.rowset, blk.c1[3], blk.arena, blk.p1, groups=groups)
        blk.p1_done[idx] = True

    def decode_rows(self, b, blk: _Block, idx, binned_t=None):
        self.block_pass1_consts(b, blk)
        self._wait_gathers(blk)
        if binned_t is None:
            binned = idx[blk.grows.binned[idx]]
            binned_t = D.h2d(binned.astype(np.int32), None, self.device) if binned.size else None
        if binned_t is not None:
            D.decode_bins(blk.grows, blk.arena, blk.cnt, order=binned_t)

    def next_block(self, extra=None):
        """The unprocessed block that completes first (the order blocks are processed in); `extra`: a block being
        opened (after the open ones)."""
        eff, oo = self.eff_hi, self.open_order
        cand = [(eff[b], 0, oo.index(b), b) for b in self.opened]
        if extra is not None:
            cand.append((eff[extra], 0, len(oo), extra))
        cand += [(eff[b], 1, k, b) for k, b in enumerate(self.pending)]
        return min(cand)[3] if cand else None

    # ---- the frame loop: wedges of consecutive frame numbers
    def feed(self, w):
        """Gathers wedge w into every open block (opening the blocks it reaches first); returns the blocks it
        completed, in processing order (each to be processed before the next block's pass 1)."""
        p = self.plan
        f, f_b = self.wedges[w]
        fi_a, fi_b = f - 1, f_b - 1
        t0 = time.perf_counter()
        while self.pending and p.need_lo[self.pending[0]] <= fi_b:
            b = self.pending.pop(0)
            blk = self.prepared.pop(b, None) or self._prepare(b)
            blk.allocate(self.device, self.f_range[0], self.eff_hi[b], self.any_excluded)
            if self.early_rows and self.next_block(extra=b) == b:
                self.block_pass1_consts(b, blk)
            self.opened[b] = blk
            self.open_order.append(b)
        t0 = self._clock("open", t0)
        ok = self.oks[w]
        ok_t = None
        if not ok.all():
            ok_t = self.ok_dev[self.ok_off:self.ok_off + ok.size]
            self.ok_off += ok.size
        if self.gs is None:
            self._gather_wedge(w, ok, ok_t, fi_a, fi_b)
        else:
            # the gathers go to the gather stream, after everything queued so far on the compute stream (block
            # openings, uploads); passes wait for the event of the wedge that completed their block
            ev = torch.cuda.Event()
            ev.record()
            self.gs.wait_event(ev)
            with torch.cuda.stream(self.gs):
                self._gather_wedge(w, ok, ok_t, fi_a, fi_b)
                ev_w = torch.cuda.Event()
                ev_w.record(self.gs)
            self.last_gathered = ev_w             # the wedge's gathers (a scheduler's latency clock waits for them)
            for b in self.opened:
                if w in self.opened[b].w_gather:
                    self.opened[b].gathered = ev_w
        if self.feeder is not None:
            self.feeder.done_with(w)
        self._clock("gather_launch", t0)
        done = sorted((b for b in self.open_order if b in self.opened and self.eff_hi[b] <= fi_b
                       and b not in self.reported), key=lambda b: (self.eff_hi[b], self.open_order.index(b)))
        self.reported.update(done)
        return done

    def _wait_gathers(self, blk):
        """The compute stream waits for the block's gathers (two-stream mode)."""
        ev = getattr(blk, "gathered", None)
        if ev is not None:
            torch.cuda.current_stream().wait_event(ev)

    def _gather_wedge(self, w, ok, ok_t, fi_a, fi_b):
        f, f_b = self.wedges[w]
        src = self.src
        if ok.any() and self.opened and self.graphs:
            data, is_f = (self.feeder.get(w), False) if self.feeder is not None else src.wedge(f, f_b, ok)
            slots = tuple(b for b in self.open_order if b in self.opened)
            if self._gg is None or self._gg.key != slots:
                blks = [self.opened[b] for b in slots]
                self._gg = D.GatherGraph(slots, [k.grows for k in blks], [k.arena for k in blks],
                                         [k.cnt for k in blks], self.device)
            steps = []
            for b in slots:
                blk = self.opened[b]
                stp = N.XiGatherStep()
                if w in blk.w_gather:
                    nf = min(fi_b, self.eff_hi[b]) - fi_a + 1
                    stp.frames = D.frames_struct(data[:nf], fi_a, None if is_f else src.overload,
                                                 0 if is_f else src.min_valid, self.mask_t,
                                                 ok_t[:nf] if ok_t is not None else None)
                    order = blk.sched(blk.w_gather[w])
                    stp.order = N.ptr(order)
                    stp.n_order = int(order.numel())
                steps.append(stp)
            self._gg.replay(steps)
        elif ok.any() and self.opened:
            data, is_f = (self.feeder.get(w), False) if self.feeder is not None else src.wedge(f, f_b, ok)
            for b in self.open_order:
                blk = self.opened.get(b)
                if blk is None or w not in blk.w_gather:
                    continue
                nf = min(fi_b, self.eff_hi[b]) - fi_a + 1
                fs = D.frames_struct(data[:nf], fi_a, None if is_f else src.overload, 0 if is_f else src.min_valid,
                                     self.mask_t, ok_t[:nf] if ok_t is not None else None)
                D.gather(fs, blk.grows, blk.sched(blk.w_gather[w]), blk.arena, blk.cnt)

    def start_pass(self, k):
        """Starts pass k over the frames (k >= 1; the blocks of the passes before it are all processed)."""
        if self.opened or self.live:
            raise RuntimeError("a pass starts after every block of the previous pass is processed")
        self.pass_index = k
        self.pending = sorted(self.passes[k], key=lambda b: self.plan.need_lo[b])
        self.prepared = {}
        self.ok_off = 0
        self._gg = None
        if self.feeder is not None:
            self.feeder.close()
            self.feeder = self.src.feeder(self.wedges, self.oks)

    def remaining(self):
        """The open blocks left after the last wedge, in processing order."""
        out = [b for b in self.open_order if b in self.opened and b not in self.reported]
        self.reported.update(out)
        return out

    def early_pass1(self, w):
        """Pass 1 of the next block's rows whose last frame arrived with wedge w (uploaded frames only; after the
        blocks wedge w completed are processed)."""
        nxt = self.next_block()
        if nxt is not None and nxt in self.opened and w in self.opened[nxt].w_early:
            blk = self.opened[nxt]
            idx, groups, bin_on = blk.w_early[w]
            idx = idx[~blk.p1_done[idx]]
            if idx.size == blk.w_early[w][0].size:          # none of them done yet: the precomputed launches apply
                self.pass1_rows(nxt, blk, idx, [(bx, dz, blk.sched(o)) for bx, dz, o in groups],
                                blk.sched(bin_on) if bin_on is not None else None)

    # ---- a completed block
    def process(self, b):
        self.pass1_stage(b)
        self.learn(b)
        self.pass2_stage(b)
        self.collect(b)

    def pass1_stage(self, b, batched=False):
        """Bin decode and pass 1 of the block's rows not done yet; batched: no launch, returns (set entry, local rows)
        for a batched launch (the caller launches, then calls learn)."""
        t0 = time.perf_counter()
        blk = self.opened.pop(b)
        self.live[b] = blk
        self._wait_gathers(blk)
        self.tg = time.time()
        self.processed.append(b)
        rem = np.flatnonzero(~blk.p1_done)
        if not batched:
            if rem.size:
                self.pass1_rows(b, blk, rem)
            self._clock("pass1_stage", t0)
            return None
        self.decode_rows(b, blk, rem)
        blk.p1_done[rem] = True
        det = self.detector(self.exp_blocks[b].geom)
        self._clock("pass1_stage", t0)
        return D.rowset_entry(det, blk.rowset, blk.c1[3], blk.arena, blk.p1), rem

    def learn(self, b):
        """Profiles and widths of a block whose pass 1 is complete: accumulation, the host adaptation (sigma_M,
        rocking-curve weights for this block's pass 2, sigma_D for the next block), finalisation."""
        t0 = time.perf_counter()
        blk = self.live[b]
        p, rs, device = self.plan, blk.rowset, self.device
        g = self.exp_blocks[b].geom
        sd_b, sm_b, rcw_b = blk.c1[:3]
        widths_p1 = (float(sd_b), float(sm_b), np.asarray(rcw_b, np.float32).copy())
        p1 = blk.p1
        num = torch.zeros((self.nreg, PROFILE_GRID, PROFILE_GRID), dtype=torch.float64, device=device)
        den = torch.zeros_like(num)
        if self.learn_profiles:
            D.accumulate(rs, p1, self.nreg, num, den)
        t0 = self._clock("learn_other", t0)
        self.prepare_ahead()                               # host work while pass 1 of the block runs
        t0 = time.perf_counter()
        h1 = _host_rows(p1.t, ADAPT_KEYS)
        t0 = self._clock("learn_wait", t0)                 # pass 1 of the block runs meanwhile
        rows = blk.rows
        if self.adaptive:
            st = _adapt_rows(h1, p, rows)
            strong = None
            if st.any():
                rst = rows[st]
                strong = dict(F=_fz_rows(p1, rs, np.flatnonzero(st)), phi=self.refl["phi"][rst],
                              zeta_k=self.refl["zeta_k"][rst], iz0=p.iz0[rst], m_d=h1["m_d"][st],
                              x=self.refl["x"][rst], y=self.refl["y"][rst])
            sm_b, rcw_b, sd_next, params = A.adapt_block(g, strong, self.sd, self.sm, sd_b, sm_b, rcw_b)
            if sd_next is not None:
                self.state.update(sd=sd_next, sm=float(sm_b), rcw=np.asarray(rcw_b, np.float32))
            self.block_params[b] = params
        t0 = self._clock("adapt", t0)
        blk.prof = torch.empty((self.nreg, PROFILE_GRID, PROFILE_GRID), dtype=torch.float32, device=device)
        D.finalize_profiles(num, den, blk.prof)
        self.block_widths[b] = dict(pass1=widths_p1,
                                    pass2=(float(sd_b), float(sm_b), np.asarray(rcw_b, np.float32).copy()))
        blk.c2 = D.block_consts(g, sd_b, sm_b, self.model.gain, rcw_b, device)
        blk.p2 = None if self.moments_only else D.Pass2Buffers(rs)
        self._clock("learn_other", t0)

    def pass2_stage(self, b, batched=False):
        """Pass 2 of the block (none for moments-only runs); batched: its set entry for a batched launch."""
        blk = self.live[b]
        if self.moments_only:
            return None
        det = self.detector(self.exp_blocks[b].geom)
        if batched:
            return D.rowset_entry(det, blk.rowset, blk.c2[0], blk.arena, blk.p1, blk.prof, blk.p2)
        t0 = time.perf_counter()
        D.pass2(det, blk.rowset, blk.c2[0], blk.arena, blk.prof, blk.p1, blk.p2)
        self._clock("pass2_stage", t0)
        return None

    def collect(self, b):
        """The block's results to the host: copies into pinned host memory queued behind pass 2 (the host goes on with
        the next wedges while pass 2 runs), put into the run's output columns once they have landed (`finish`). The
        block's arena goes back to the pool now: its next user writes it on this stream, after every kernel that
        reads it (unless a captured gather graph still names it)."""
        t0 = time.perf_counter()
        blk = self.live.pop(b)
        p1, rs = blk.p1, blk.rowset
        cols = {k: p1.t[k] for k in P1_OUT}
        if blk.p2 is not None:
            cols.update({k: blk.p2.t[k] for k in P2_OUT})
        c = _Collected(b, blk.rows, blk.span, blk.rows_sorted, self.tg)     # no device buffer kept past the copies
        c.host = _host_rows_async(cols, tuple(cols), blk.perm_t)
        c.prof = _pinned_copy(blk.prof)
        if self.fz_out is not None:
            c.fz = _pinned_copy(_fz_rows(p1, rs, np.arange(rs.n)).float())
        c.status = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        N.check(N.load().xi_status_copy(c.status.data_ptr(), N.stream_handle()), "xi_status_copy")
        c.ev = torch.cuda.Event()
        c.ev.record()
        self.collects.append(c)
        if self._gg is None or b not in self._gg.key:
            D.POOL.give(blk.arena)
            blk.arena = None
        p1.release()
        self._clock("collect", t0)
        self.finish(wait=False)

    def finish(self, wait=True):
        """Collected blocks whose copies have landed (every one: wait) into the run's output columns, in order."""
        while self.collects:
            c = self.collects[0]
            if not wait and not c.ev.query():
                return
            t0 = time.perf_counter()
            c.ev.synchronize()
            self.collects.pop(0)
            if int(c.status[0]):
                D.status()                                  # reports (raises) and clears the status word
            self.prof_by_block[c.b] = c.prof.numpy()
            dst = slice(*c.span) if c.span is not None else c.rows_sorted
            for k, v in c.host.items():
                self.out[k][dst] = v.numpy()
            if c.fz is not None:
                self.fz_out[c.rows] = c.fz.numpy()
            self.t_dev += time.time() - c.tg
            self._clock("finish", t0)

    def _clock(self, stage, t0):
        """Adds the host seconds since t0 to the stage's total; returns the time now."""
        t = time.perf_counter()
        self.host_s[stage] = self.host_s.get(stage, 0.0) + t - t0
        return t

    def result(self):
        self.finish()
        t0 = time.perf_counter()
        p, out, refl = self.plan, self.out, self.refl
        unfilled = np.ones(p.n, bool)                     # rows of blocks never processed: NaN, as XPG leaves them
        for b in self.processed:
            unfilled[p.blocks_refl[b]] = False
        for k in OUT_F64:
            if self.moments_only and k not in P1_OUT:     # pass 2 did not run
                out[k][:] = np.nan
            else:
                out[k][unfilled] = np.nan
        refl.update(out)
        refl["overlap"] = p.overlap
        if self.fz_out is not None:
            refl["fz"] = self.fz_out
        refl["iz0"], refl["dz"], refl["fb"] = p.iz0, p.dz, p.fb
        refl["region"] = p.region
        refl["ix0"], refl["iy0"] = p.ix0 * p.pxs, p.iy0 * p.pxs
        if (p.pxs > 1).any():
            refl["pxs"] = p.pxs
        if self.verbose:
            okk = np.isfinite(refl["iprf"])
            self.log(f"  INTEGRATE: {okk.sum()} reflections integrated in {time.time() - self.t0:.1f}s "
                     f"(device {self.t_dev:.1f}s)")
        self._clock("result", t0)
        res = IntegrationResult(refl, self.model, self.prof_by_block, dict(total=time.time() - self.t0,
                                                                           gpu=self.t_dev,
                                                                           host_s=dict(self.host_s)))
        res.block_params = self.block_params
        res.block_widths = self.block_widths  # (sigma_D, sigma_M in radians, rocking-curve weights) of each pass
        res.plan = self.plan                  # the plan integrated (blocks split in parts when memory was short)
        res.block_order = list(self.processed)  # blocks (of res.plan) in the order they were processed
        res.memory = self.mem
        return res

    def close(self):
        if self.feeder is not None:
            self.feeder.close()
            self.feeder = None
        self._gg = None
        if self.src is not None and getattr(self.src, "_buf", None) is not None:
            D.POOL.give(self.src._buf)
            self.src._buf = None
        if not D.POOL.persist:
            D.POOL.clear()                    # the kept arenas go back to the allocator between runs
            torch.cuda.empty_cache()          # and to the device: the next run's small buffers must not split them


ADAPT_KEYS = ("isum", "vsum", "n_over", "frac_rec", "m_d")
P1_OUT = ("bg", "isum", "vsum", "vsum0", "xo", "yo", "zo", "frac_rec", "m_d", "m_m", "n_over", "n_fg_masked",
          "isum_raw")
P2_OUT = ("iprf", "vprf", "vprf0", "corr", "p_valid", "p_total", "rho", "p_fg")


class _Collected:
    """A block's results on their way to the host: pinned copies queued on the compute stream, the kernels' status
    word, and an event after them."""

    def __init__(self, b, rows, span, rows_sorted, tg):
        self.b, self.rows, self.span, self.rows_sorted, self.tg = b, rows, span, rows_sorted, tg
        self.host, self.prof, self.fz, self.status, self.ev = {}, None, None, None, None


def _pinned_copy(t):
    """Queues a copy of device tensor t into new pinned host memory on the current stream (read after a sync)."""
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t, non_blocking=True)
    return h


def _host_rows_async(t, keys, perm=None):
    """`_host_rows` without waiting: one stacked pinned copy per dtype queued on the current stream; values are host
    tensor rows, valid once the stream has passed the copies."""
    out = {}
    for dt in (torch.float32, torch.int64):
        ks = [k for k in keys if t[k].dtype == dt]
        if not ks:
            continue
        st = torch.stack([t[k] for k in ks])
        if perm is not None:
            st = st.index_select(1, perm)
        h = _pinned_copy(st)
        out.update({k: h[i] for i, k in enumerate(ks)})
    return out


def _host_rows(t, keys, perm=None):
    """Per-row device outputs on the host (`xpg/integrate_kernels.py:169-183`), optionally permuted on the device
    first: one stacked copy per dtype."""
    out = {}
    for dt in (torch.float32, torch.int64):
        ks = [k for k in keys if t[k].dtype == dt]
        if not ks:
            continue
        st = torch.stack([t[k] for k in ks])
        if perm is not None:
            st = st.index_select(1, perm)
        st = D.d2h(st)
        out.update({k: st[i] for i, k in enumerate(ks)})
    return out


def _fz_rows(p1: D.Pass1Buffers, rs: D.RowSet, rows):
    """fz of the given local rows, padded to the deepest box with zeros: a (n, 65) float64 device tensor."""
    if rows.size == 0:
        return torch.zeros((0, MAX_DZ), dtype=torch.float64, device=rs.device)
    r = D.h2d(rows, None, rs.device)
    k = torch.arange(MAX_DZ, device=rs.device)
    off = rs.t["frm_off"].index_select(0, r)[:, None] + k
    ok = k[None] < rs.t["Dz"].index_select(0, r)[:, None]
    return torch.where(ok, p1.t["fz"][torch.where(ok, off, 0)], torch.zeros((), device=rs.device)).double()


def _adapt_rows(h1, plan, rows):
    """Strong rows of the per-block adaptation (`xpg/integrate.py:411-414`), float64 on the float32 outputs. The
    integer tests go first; the float64 ratio is evaluated on the rows that pass them only (same arithmetic per row)."""
    fb = plan.fb[rows[0]:rows[-1] + 1] if rows.size and rows[-1] - rows[0] + 1 == rows.size else plan.fb[rows]
    cand = np.flatnonzero((h1["n_over"] == 0) & (fb == 1) & (h1["isum"] > 0))
    isum = h1["isum"][cand].astype(np.float64)
    vs = h1["vsum"][cand].astype(np.float64)
    ok = (isum / np.sqrt(np.maximum(vs, 1e-6)) > 15) & (h1["frac_rec"][cand].astype(np.float64) > 0.98)
    st = np.zeros(rows.size, bool)
    st[cand[ok]] = True
    return st


def estimate_sigmas(images, exp, model0: IntegrationModel, dmin, frames, n_sample_frames=30, verbose=True, log=print,
                    extra_exps=(), bkg_template=None, foreign_spots=None, max_iter=None, guard=None):
    """sigma_D / sigma_M from strong spots (`xpg/integrate.py:1002-1092`), on moments-only device integrations."""
    return A.estimate_sigmas(integrate, images, exp, model0, dmin, frames, n_sample_frames, verbose, log, extra_exps,
                             bkg_template, foreign_spots, max_iter, guard)
