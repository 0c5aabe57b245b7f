"""Device-side objects of the integration path: detector constants, packed per-reflection rows, the shoebox arena
and the pass outputs, each with the C struct that the kernels read (include/xpgi.h).

Every buffer is a torch CUDA tensor (torch is the allocator and the stream); the arithmetic runs in libxpgi.so.
"""
from __future__ import annotations

import collections
import ctypes as C
import functools
import threading

import numpy as np
import torch

from . import native as N

F32 = torch.float32


class KernelTimer:
    """Optional per-kernel CUDA-event timing of the library calls (pairs of events on the launching stream around
    each call) and a count of kernel launches. Off unless `TIMER.enabled`; read after a synchronize."""

    def __init__(self):
        self.enabled = False
        self.reset()

    def reset(self):
        self.events = []                 # (name, start, end)
        self.launches = 0

    def span(self, name, n_launches=1):
        return _Span(self, name, n_launches)

    def summary(self):
        out = {}
        for name, a, b in self.events:
            t = a.elapsed_time(b) * 1e-3
            d = out.setdefault(name, [0, 0.0])
            d[0] += 1
            d[1] += t
        return out


class _Span:
    def __init__(self, timer, name, n):
        self.t, self.name, self.n = timer, name, n

    def __enter__(self):
        self.t.launches += self.n
        if self.t.enabled:
            self.a = torch.cuda.Event(enable_timing=True)
            self.a.record()
        return self

    def __exit__(self, *exc):
        if self.t.enabled:
            b = torch.cuda.Event(enable_timing=True)
            b.record()
            self.t.events.append((self.name, self.a, b))
        return False


TIMER = KernelTimer()


class _UploadRing:
    """Page-locked staging ring of the uploads, allocated once per process. An upload is copied into the ring and
    read from there by a kernel on the current stream (xi_upload), not by the copy engine: that serves copies in
    submission order, so a small upload would otherwise wait behind every frame chunk already queued. A region is
    rewritten only after the kernel that read it has run (regions are taken in ring order, so the ones a new region
    overlaps are the oldest in flight); while they have not run, the upload takes the copy engine instead, so the
    host never waits for the device here."""

    SIZE = 256 << 20

    def __init__(self):
        self.buf = None
        self.head = 0
        self.inflight = collections.deque()      # (start, end, event), oldest first
        self.lock = threading.Lock()

    def upload(self, t, out, stream):
        """Copies CPU tensor t into device tensor out on `stream`; False when t does not fit or the ring's memory is
        not mapped into the device (the caller copies another way)."""
        n = t.numel() * t.element_size()
        size = (n + 255) // 256 * 256
        if size > self.SIZE // 4:
            return False
        with self.lock:
            if self.buf is None:
                self.buf = torch.empty(self.SIZE, dtype=torch.uint8, pin_memory=True)
            a = self.head if self.head + size <= self.SIZE else 0
            b = a + size
            while self.inflight and self.inflight[0][0] < b and self.inflight[0][1] > a:
                if not self.inflight[0][2].query():
                    return False
                self.inflight.popleft()
            base = self.buf.data_ptr()
            C.memmove(base + a, t.data_ptr(), n)
            rc = N.load().xi_upload(C.c_void_p(base + a), C.c_void_p(out.data_ptr()), n, C.c_void_p(stream.cuda_stream))
            if rc != N.XI_OK:
                return False
            ev = torch.cuda.Event()
            ev.record(stream)
            self.inflight.append((a, b, ev))
            self.head = b
            return True


_RING = _UploadRing()


class BufferPool:
    """Large device buffers kept across uses: the shoebox arenas of successive blocks (tens of GB each) and frame
    wedges. The caching allocator splits and fragments such blocks when they are freed and allocated block after
    block; here a request takes the smallest kept buffer that holds it (a view of its first elements) if that is at
    most FIT times the request (a small block holding a large buffer would leave the next large block to allocate
    anew, beyond what the memory plan counts), else a new one allocated SLACK larger than asked (so that later blocks
    of about the same size fit), and `give` returns it. A buffer is given back once every kernel that uses it is
    queued: `give` records an event on the giver's stream, the next taker's stream waits for it, and the taker's
    stream is recorded on the buffer (so that the allocator keeps it until that stream's work is done when it is
    freed), which keeps reuse safe across the streams of several host threads."""

    SLACK = 1.05
    FIT = 1.3
    KEEP = 2

    def __init__(self):
        self.free = {}                 # (device index, dtype) -> [tensor]
        self.persist = False           # kept buffers outlive a run (keep_buffers)
        self.lock = threading.RLock()  # sweeps integrated on several host threads share the pool
        self.ready = {}                # id(buffer) -> event recorded when it was given back

    def take(self, n, dtype, device):
        with self.lock:
            return self._take(n, dtype, device)

    def _take(self, n, dtype, device):
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        key = (dev.index, dtype)
        pool = self.free.setdefault(key, [])
        fits = [i for i, t in enumerate(pool) if n <= t.numel() <= self.FIT * n + 4096]
        if fits:
            i = min(fits, key=lambda j: pool[j].numel())
            base = pool.pop(i)
            ev = self.ready.pop(id(base), None)
            if base.is_cuda:
                st = torch.cuda.current_stream(base.device)
                if ev is not None:
                    st.wait_event(ev)
                base.record_stream(st)
            return base[:n]
        for t in pool:                                    # kept buffers too small for this request: memory back first
            if t.numel() <= n:
                self.ready.pop(id(t), None)
        pool[:] = [t for t in pool if t.numel() > n]
        size = max(int(n * self.SLACK), 1)
        try:
            return torch.empty(size, dtype=dtype, device=dev)[:n]
        except torch.OutOfMemoryError:
            for t in pool:
                self.ready.pop(id(t), None)
            pool.clear()                # the kept buffers: let the allocator have their memory
            torch.cuda.empty_cache()
            return torch.empty(n, dtype=dtype, device=dev)

    def retain(self, wanted):
        """Keeps only the kept buffers that one of the requests `wanted` ({dtype: [element counts]}) would take; the
        others go back to the device (a run whose buffers differ in size from the last run's)."""
        with self.lock:
            self._retain(wanted)

    def _retain(self, wanted):
        dropped = False
        for (_, dt), pool in self.free.items():
            sizes = wanted.get(dt, ())
            keep = [t for t in pool if any(n <= t.numel() <= self.FIT * n + 4096 for n in sizes)]
            for t in pool:
                if not any(t is k for k in keep):
                    self.ready.pop(id(t), None)
            if len(keep) != len(pool):
                pool[:] = keep
                dropped = True
        if dropped:
            torch.cuda.empty_cache()

    def give(self, t):
        if t is None:
            return
        with self.lock:
            self._give(t)

    def _give(self, t):
        base = t._base if t._base is not None else t
        key = (base.device.index, base.dtype)
        pool = self.free.setdefault(key, [])
        if not any(x is base for x in pool):
            pool.append(base)
            if base.is_cuda:
                ev = torch.cuda.Event()
                ev.record(torch.cuda.current_stream(base.device))
                self.ready[id(base)] = ev
        pool.sort(key=lambda x: -x.numel())
        for x in pool[self.KEEP:]:
            self.ready.pop(id(x), None)
        del pool[self.KEEP:]

    def clear(self):
        with self.lock:
            self.free.clear()
            self.ready.clear()


POOL = BufferPool()


def keep_buffers(on=True):
    """Keeps the pooled device buffers (shoebox arenas, pass-1 tables, frame wedges; tens of GB) from one
    integration to the next, for callers that integrate sweep after sweep on a device of their own: the next run
    takes them instead of allocating anew. Off by default: a run then gives its buffers and the allocator's cached
    memory back to the device when it returns. `keep_buffers(False)` also releases what is kept."""
    POOL.persist = bool(on)
    if not on:
        POOL.clear()
        torch.cuda.empty_cache()


def h2d(a, dtype=None, device="cuda"):
    """Host array -> device tensor on the current stream without blocking the host: staged through the upload ring
    and read by a kernel (large arrays: through torch's pinned staging and the copy engine). A pageable copy would
    wait for every kernel queued before it."""
    a = np.ascontiguousarray(a)
    if not a.flags.writeable:                 # torch does not wrap read-only arrays (a broadcast view, a plan column)
        a = a.copy()
    t = torch.as_tensor(a, dtype=dtype)
    if t.numel() == 0:
        return t.to(device)
    t = t.contiguous()
    out = torch.empty(t.shape, dtype=t.dtype, device=device)
    if _RING.upload(t, out, torch.cuda.current_stream(out.device)):
        return out
    out.copy_(t.pin_memory(), non_blocking=True)
    return out


def d2h(t):
    """Device tensor -> host numpy array through pinned memory (the array keeps its pinned block alive)."""
    if t.numel() == 0:
        return t.cpu().numpy()
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t)
    return h.numpy()


def _dev(a, dtype, device):
    if torch.is_tensor(a):                  # already a tensor (the planner's device columns): convert in place
        return a.to(device=device, dtype=dtype).contiguous()
    return h2d(a, dtype, device)


class DeviceDetector:
    """XPG's `_detector_consts` (`xpg/integrate_kernels.py:48-65`) on the device."""

    def __init__(self, g, bkg_template=None, device="cuda"):
        P0, Bx, By = g.panels()
        U1, U2 = Bx / g.qx, By / g.qy
        UN = np.cross(U1, U2)
        f = lambda a: _dev(np.asarray(a, np.float32).reshape(-1, 3), F32, device)
        self.t = dict(P0=f(P0), Bx=f(Bx), By=f(By), U1=f(U1), U2=f(U2), UN=f(UN))
        seg = g.segmap() if getattr(g, "segmented", False) else None
        geo = getattr(g, "geo_corr", None)
        self.t["segmap"] = None if seg is None else _dev(seg.astype(np.int16), torch.int16, device)
        self.t["gx"] = None if geo is None else _dev(np.asarray(geo[0], np.float32), F32, device)
        self.t["gy"] = None if geo is None else _dev(np.asarray(geo[1], np.float32), F32, device)
        self.t["bkg"] = None if bkg_template is None else _dev(np.asarray(bkg_template, np.float32), F32, device)
        d = N.XiDetector()
        d.n_panels = int(np.asarray(P0).reshape(-1, 3).shape[0])
        for k in ("P0", "Bx", "By", "U1", "U2", "UN", "segmap", "gx", "gy", "bkg"):
            setattr(d, k, N.ptr(self.t[k]))
        if seg is not None:
            d.seg_ny, d.seg_nx = seg.shape
        if geo is not None:
            d.geo_ny, d.geo_nx = np.asarray(geo[0]).shape
        if bkg_template is not None:
            d.bkg_ny, d.bkg_nx = np.asarray(bkg_template).shape
        d.orgx, d.orgy = float(g.orgx), float(g.orgy)
        d.qx, d.qy, d.wl = float(g.qx), float(g.qy), float(g.wavelength)
        tsens = float(max(g.sensor_thickness, 1e-6))
        mu = float(max(g.mu, 1e-6))
        d.tsens, d.mu, d.inv_mu = tsens, mu, 1.0 / mu
        d.parallax = 1 if g.has_parallax else 0
        self.s = d


def block_consts(g, sd, sm, gain, rcw, device="cuda"):
    """XiBlock of a phi block (`xpg/integrate.py:466-475`): returns (struct, keep-alive tensors)."""
    b = N.XiBlock()
    b.frames_phi0 = float(np.float32(np.radians(g.z_to_phi(0.0))))
    b.osc = float(np.float32(np.radians(g.osc)))
    b.sd, b.sm, b.gain = float(np.float32(sd)), float(np.float32(sm)), float(np.float32(gain))
    rc = _dev(np.asarray(rcw, np.float32), F32, device)
    b.rcw = N.ptr(rc)
    s0 = np.asarray(g.s0, np.float32)
    ax = np.asarray(g.axis, np.float32)
    for c in range(3):
        b.s0[c] = float(s0[c])
        b.axis[c] = float(ax[c])
    return b, rc


def _offsets(sizes):
    """Exclusive prefix sum (int64): where each row's block starts."""
    out = np.zeros(sizes.size, np.int64)
    if sizes.size > 1:
        np.cumsum(sizes[:-1], out=out[1:])
    return out


class RowSet:
    """Per-reflection inputs of a set of rows (any mix of shoebox shapes), packed on the device with their arena
    offsets: `sb_off` (shoebox voxels), `pix_off` (per-pixel outputs), `frm_off` (per-frame outputs)."""

    def __init__(self, S, phi, ix0, iy0, iz0, fb, region, has_p, pS, pphi, pxs, Dz, bx, nb, device="cuda",
                 sb_bias=3.0):
        n = len(phi)
        self.n = n
        self.Dz = np.asarray(Dz, np.int64)
        self.bx = np.asarray(bx, np.int64)
        self.sb_bias = sb_bias
        P = self.bx * self.bx
        self.n_vox = int(self._vp(self.Dz * P).sum()) + 4
        self.n_pix = int(P.sum())
        self.n_frm = int(self.Dz.sum())
        K = int(nb["x"].shape[1]) if n else 0
        if K > N.XI_MAX_K:
            raise ValueError(f"{K} neighbour columns > {N.XI_MAX_K}")
        d = device
        dzbx = _dev(np.stack([self.Dz, self.bx]), torch.int32, d)      # one upload for both
        dz64, bx64 = dzbx[0].long(), dzbx[1].long()
        p64 = bx64 * bx64
        vp64 = self._vp(dz64 * p64)
        self.t = dict(
            S=_dev(S, F32, d).reshape(n, 3), phi=_dev(phi, F32, d),
            ix0=_dev(ix0, torch.int32, d), iy0=_dev(iy0, torch.int32, d), iz0=_dev(iz0, torch.int32, d),
            fb=_dev(fb, F32, d), region=_dev(region, torch.int32, d),
            has_p=_dev(has_p, F32, d), pS=_dev(pS, F32, d).reshape(n, 3),
            pphi=_dev(pphi, F32, d), pxs=_dev(pxs, torch.int32, d), Dz=dzbx[0], bx=dzbx[1],
            sb_off=torch.cumsum(vp64, 0) - vp64, pix_off=torch.cumsum(p64, 0) - p64,
            frm_off=torch.cumsum(dz64, 0) - dz64)
        for k in ("x", "y", "z", "sx", "sz"):
            self.t["nb" + k] = _dev(nb[k], F32, d).reshape(n, K)
        r = N.XiRows()
        r.n = n
        for k in ("S", "phi", "ix0", "iy0", "iz0", "fb", "region", "has_p", "pS", "pphi", "pxs", "Dz", "bx",
                  "sb_off", "pix_off", "frm_off", "nbx", "nby", "nbz", "nbsx", "nbsz"):
            setattr(r, k, N.ptr(self.t[k]))
        r.K = K
        r.order = None
        r.n_order = 0
        r.max_bx = int(self.bx.max()) if n else 3
        r.max_dz = int(self.Dz.max()) if n else 1
        r.sb_bias = float(sb_bias)
        self.s = r
        self.device = device

    def _vp(self, v):
        """Arena floats of rows of v voxels: with the +3 encoding every row starts on 16 bytes (bulk copies)."""
        return (v + 3) & ~3 if self.sb_bias == 3.0 else v

    @functools.cached_property
    def vox(self):
        return self.Dz * self.bx * self.bx

    @functools.cached_property
    def sb_off(self):
        return _offsets(self._vp(self.vox))

    @functools.cached_property
    def pix_off(self):
        return _offsets(self.bx * self.bx)

    @functools.cached_property
    def frm_off(self):
        return _offsets(self.Dz)

    def groups(self):
        """Launch groups: rows of one shoebox shape (side, depth), so that each launch sizes its shared memory
        (and decides whether the shoebox is staged there) for exactly its rows. Largest shapes first."""
        out = []
        if self.n == 0:
            return out
        key = self.bx * 128 + self.Dz
        order = np.argsort(key, kind="stable")
        uk, start = np.unique(key[order], return_index=True)
        stop = np.append(start[1:], order.size)
        for k, a, e in zip(uk, start, stop):
            out.append((int(k // 128), int(k % 128), order[a:e].astype(np.int32)))
        out.sort(key=lambda g: -g[0] * g[0] * g[1])
        return out

    def view(self, order=None, max_bx=None, max_dz=None):
        """A copy of the struct restricted to `order` (device int32 tensor) with its shape maxima."""
        r = N.XiRows.from_buffer_copy(self.s)
        if order is not None:
            r.order = N.ptr(order)
            r.n_order = int(order.numel())
        if max_bx is not None:
            r.max_bx = int(max_bx)
        if max_dz is not None:
            r.max_dz = int(max_dz)
        return r


class Pass1Buffers:
    """Pass-1 outputs of a RowSet (`xpg/integrate_kernels.py:362-365`)."""

    SCALARS = ("bg", "nbg", "isum", "vsum", "vsum0", "xo", "yo", "zo", "m_d", "m_m", "frac_rec", "nfg", "zeta",
               "seff")
    COUNTS = ("n_over", "n_fg_masked", "n_fg_nb", "isum_raw")

    def __init__(self, rows: RowSet, pooled=False):
        """pooled: the per-pixel tables (17 bytes a pixel, GBs for a block) as views of one buffer from POOL, given
        back by `release` (the caching allocator would otherwise split the large blocks it keeps for them)."""
        d = rows.device
        n = rows.n
        self.t = {k: torch.empty(n, dtype=F32, device=d) for k in self.SCALARS}
        self.t.update({k: torch.empty(n, dtype=torch.int64, device=d) for k in self.COUNTS})
        self.t["fz"] = torch.empty(rows.n_frm, dtype=F32, device=d)
        self.base = None
        if pooled:
            step = (rows.n_pix * 4 + 255) // 256 * 256              # each table on 256 bytes
            self.base = POOL.take(4 * step + max(rows.n_pix, 1), torch.uint8, d)
            for i, k in enumerate(("img2", "J", "u1", "u2")):
                self.t[k] = self.base[i * step:i * step + rows.n_pix * 4].view(F32)
            self.t["all_valid2"] = self.base[4 * step:4 * step + rows.n_pix]
        else:
            for k in ("img2", "J", "u1", "u2"):
                self.t[k] = torch.empty(rows.n_pix, dtype=F32, device=d)
            self.t["all_valid2"] = torch.empty(rows.n_pix, dtype=torch.uint8, device=d)
        o = N.XiPass1Out()
        for k, v in self.t.items():
            setattr(o, k, N.ptr(v))
        self.s = o

    def release(self):
        """The pooled per-pixel tables back to POOL (their next user writes them in stream order)."""
        if self.base is not None:
            POOL.give(self.base)
            self.base = None
            for k in ("img2", "J", "u1", "u2", "all_valid2"):
                self.t.pop(k, None)

    def pass2_in(self):
        i = N.XiPass2In()
        for k in ("zeta", "seff", "J", "u1", "u2", "bg", "nbg"):
            setattr(i, k, N.ptr(self.t[k]))
        return i


class Pass2Buffers:
    KEYS = ("iprf", "vprf", "vprf0", "corr", "p_valid", "p_total", "ipartner", "rho", "p_fg")

    def __init__(self, rows: RowSet):
        self.t = {k: torch.empty(rows.n, dtype=F32, device=rows.device) for k in self.KEYS}
        o = N.XiPass2Out()
        for k, v in self.t.items():
            setattr(o, k, N.ptr(v))
        self.s = o


def _stream(stream):
    return N.stream_handle(stream)


def pass1(det: DeviceDetector, rows: RowSet, blk, arena, out: Pass1Buffers, stream=None, groups=None):
    """Pass 1 of every row, one launch per box side."""
    lib = N.load()
    for bxg, dzg, order in (groups if groups is not None else _device_groups(rows)):
        r = rows.view(order, bxg, dzg)
        with TIMER.span("pass1"):
            N.check(lib.xi_pass1(C.byref(det.s), C.byref(r), C.byref(blk), N.ptr(arena), C.byref(out.s),
                                 _stream(stream)), "xi_pass1")


def pass2(det: DeviceDetector, rows: RowSet, blk, arena, prof, p1: Pass1Buffers, out: Pass2Buffers, stream=None,
          groups=None):
    lib = N.load()
    i2 = p1.pass2_in()
    for bxg, dzg, order in (groups if groups is not None else _device_groups(rows)):
        r = rows.view(order, bxg, dzg)
        with TIMER.span("pass2"):
            N.check(lib.xi_pass2(C.byref(det.s), C.byref(r), C.byref(blk), N.ptr(arena), N.ptr(prof), C.byref(i2),
                                 C.byref(out.s), _stream(stream)), "xi_pass2")


def accumulate(rows: RowSet, p1: Pass1Buffers, n_regions, num, den, sel=None, strong_test=True, order=None,
               stream=None):
    lib = N.load()
    r = rows.view(order)
    with TIMER.span("accumulate"):
        N.check(lib.xi_accumulate(C.byref(r), C.byref(p1.s), N.ptr(sel), 1 if strong_test else 0, int(n_regions),
                                  N.ptr(num), N.ptr(den), _stream(stream)), "xi_accumulate")


def finalize_profiles(num, den, prof, stream=None):
    lib = N.load()
    with TIMER.span("finalize"):
        N.check(lib.xi_finalize_profiles(N.ptr(num), N.ptr(den), int(num.shape[0]), N.ptr(prof), _stream(stream)),
                "xi_finalize_profiles")


def status(stream=None):
    N.check(N.load().xi_status(_stream(stream)), "kernel status")


def _device_groups(rows: RowSet):
    cache = getattr(rows, "_groups", None)
    if cache is None:
        cache = [(b, dz, h2d(o, None, rows.device)) for b, dz, o in rows.groups()]
        rows._groups = cache
    return cache


class GatherRows:
    """Boxes of a block's rows for the frame gather (`xpg/integrate.py:372-398`), with bin counters for binned
    rows."""

    def __init__(self, rows: RowSet, ix0, iy0, iz0, fb, pxs, device="cuda"):
        n = rows.n
        fb = np.asarray(fb, np.int64)
        binned = fb > 1
        self.any_binned = bool(binned.any())
        self.n_cnt = int(rows.Dz[binned].sum()) if self.any_binned else 0
        d = device
        fb_t = _dev(fb, torch.int32, d)
        if self.any_binned:                  # bin counters of binned rows, packed in row order; -1 elsewhere
            bin_t = fb_t > 1
            cl = torch.where(bin_t, rows.t["Dz"].long(), 0)
            cnt_off = torch.where(bin_t, torch.cumsum(cl, 0) - cl, -1)
        else:
            cnt_off = torch.full((n,), -1, dtype=torch.int64, device=d)
        self.t = dict(ix0=_dev(ix0, torch.int32, d), iy0=_dev(iy0, torch.int32, d), iz0=_dev(iz0, torch.int32, d),
                      fb=fb_t, Dz=rows.t["Dz"], bx=rows.t["bx"], pxs=_dev(pxs, torch.int32, d),
                      sb_off=rows.t["sb_off"], cnt_off=cnt_off)
        g = N.XiGatherRows()
        g.n = n
        for k, v in self.t.items():
            setattr(g, k, N.ptr(v))
        g.order = None
        g.n_order = 0
        self.s = g
        self.span = rows.Dz * fb
        self.binned = binned

    def view(self, order):
        g = N.XiGatherRows.from_buffer_copy(self.s)
        g.order = N.ptr(order)
        g.n_order = int(order.numel())
        return g


def frames_struct(data, first_fi, overload, min_valid=0, mask=None, frame_ok=None):
    """XiFrames of a device wedge (n_frames, ny, nx) of uint32 raw counts or float32 prepared frames."""
    f = N.XiFrames()
    f.data = N.ptr(data)
    f.is_float = 1 if data.dtype == torch.float32 else 0
    if data.dtype not in (torch.float32, torch.int32, torch.uint32):
        raise TypeError("frames must be uint32 (raw) or float32 (prepared)")
    f.n_frames, f.ny, f.nx = (int(v) for v in data.shape)
    f.first_fi = int(first_fi)
    f.frame_ok = N.ptr(frame_ok)
    f.overload = int(min(int(overload), 0xFFFFFFFF)) if overload is not None else 0xFFFFFFFF
    f.min_valid = int(min_valid)
    f.mask = N.ptr(mask)
    return f


def gather(frames_s, grows: GatherRows, order, arena, cnt, stream=None):
    lib = N.load()
    g = grows.view(order)
    with TIMER.span("gather"):
        N.check(lib.xi_gather(C.byref(frames_s), C.byref(g), N.ptr(arena), N.ptr(cnt), _stream(stream)),
                "xi_gather")


def decode_bins(grows: GatherRows, arena, cnt, stream=None, order=None):
    """Decode the binned rows (all, or the device int32 `order` subset)."""
    lib = N.load()
    g = grows.s if order is None else grows.view(order)
    with TIMER.span("decode_bins"):
        N.check(lib.xi_decode_bins(C.byref(g), N.ptr(arena), N.ptr(cnt), _stream(stream)), "xi_decode_bins")


def zero_rows(grows: GatherRows, arena, order, stream=None):
    """Zeroes the arena slots of the rows in the device int32 `order` (xi_zero_rows)."""
    N.check(N.load().xi_zero_rows(C.byref(grows.view(order)), N.ptr(arena), _stream(stream)), "xi_zero_rows")


def host_groups(rows: RowSet, idx):
    """Launch groups (as RowSet.groups: one shape each, largest first) of the local rows idx, as host int32 arrays."""
    idx = np.asarray(idx, np.int64)
    if idx.size == 0:
        return []
    key = rows.bx[idx] * 128 + rows.Dz[idx]
    o = np.argsort(key, kind="stable")
    ks = key[o]
    uk, start = np.unique(ks, return_index=True)
    stop = np.append(start[1:], o.size)
    out = [(int(k // 128), int(k % 128), idx[o[a:e]].astype(np.int32)) for k, a, e in zip(uk, start, stop)]
    out.sort(key=lambda g: -g[0] * g[0] * g[1])
    return out


def subset_groups(rows: RowSet, idx):
    """Launch groups of the local rows idx, with device order tensors."""
    return [(b, dz, h2d(r, None, rows.device)) for b, dz, r in host_groups(rows, idx)]


# ---- batched passes: rows of many blocks (of many sweeps) per launch --------------------------------------------

def rowset_entry(det: DeviceDetector, rows: RowSet, blk, arena, p1: Pass1Buffers, prof=None, p2=None):
    """XiRowSet of one block's rows: its detector, constants, arena and buffers (pass 2: profiles and outputs)."""
    e = N.XiRowSet()
    e.det = det.s
    e.rows = rows.s
    e.blk = blk
    e.arena = N.ptr(arena)
    e.p1 = p1.s
    if prof is not None:
        e.prof = N.ptr(prof)
    if p2 is not None:
        e.p2 = p2.s
    return e


class RowSetTable:
    """The XiRowSet array of a batched call, in device memory."""

    def __init__(self, entries, device="cuda"):
        arr = (N.XiRowSet * len(entries))(*entries)
        self.t = h2d(np.frombuffer(bytes(arr), np.uint8), None, device)
        self.n = len(entries)
        self.k_max = max((int(e.rows.K) for e in entries), default=0)


# Size bins of a batched launch: upper bounds on the box side; a bin's launch sizes shared memory and threads for its
# largest box (the side bucket) and depth. The tuned bins of the device (xpg_b200.tune, tuned.json) replace these.
DEFAULT_BINS = (17, 31, 41, 55, 97)


def batched_items(groups, bins=None, device="cuda"):
    """Launch bins of a batched pass. groups: (set index, local rows, their sides, their depths) per set. Returns
    [(max_bx, max_dz, items)] with items an int64 device tensor (set << 32 | row), each bin's rows largest box
    first (resident CTAs take the big rows before the small ones, which balances the launch)."""
    if bins is None:
        from .tune import load_bins
        bins = load_bins() or DEFAULT_BINS
    bins = tuple(bins)
    cols = [(np.full(len(r), s, np.int64), np.asarray(r, np.int64), np.asarray(b, np.int64), np.asarray(d, np.int64))
            for s, r, b, d in groups if len(r)]
    if not cols:
        return []
    st, rw, bx, dz = (np.concatenate([c[k] for c in cols]) for k in range(4))
    if int(bx.max()) > bins[-1]:                 # sides beyond the bins (tuned on another workload): one more bin
        bins = bins + (int(bx.max()),)
    which = np.searchsorted(np.asarray(bins), bx, side="left")
    out = []
    for k in np.unique(which):
        m = np.flatnonzero(which == k)
        vol = bx[m] * bx[m] * dz[m]
        o = m[np.argsort(-vol, kind="stable")]
        items = (st[o] << 32) | rw[o]
        out.append((int(bx[m].max()), int(dz[m].max()), h2d(items, None, device)))
    return out


_QUEUES = {}


def _queue(device):
    key = torch.device(device).index if torch.device(device).index is not None else torch.cuda.current_device()
    if key not in _QUEUES:
        _QUEUES[key] = torch.zeros(64, dtype=torch.int32, device=device)
    return _QUEUES[key]


def pass1_batched(table: RowSetTable, launches, stream=None):
    """Pass 1 of every item of the launches (batched_items), one persistent launch per size bin."""
    lib = N.load()
    q = _queue(table.t.device)
    for i, (mbx, mdz, items) in enumerate(launches):
        with TIMER.span("pass1"):
            N.check(lib.xi_pass1_batched(N.ptr(table.t), N.ptr(items), int(items.numel()), mbx, mdz, table.k_max,
                                         C.c_void_p(q.data_ptr() + 4 * (i % 64)), _stream(stream)),
                    "xi_pass1_batched")


def pass2_batched(table: RowSetTable, launches, stream=None):
    lib = N.load()
    q = _queue(table.t.device)
    for i, (mbx, mdz, items) in enumerate(launches):
        with TIMER.span("pass2"):
            N.check(lib.xi_pass2_batched(N.ptr(table.t), N.ptr(items), int(items.numel()), mbx, mdz, table.k_max,
                                         C.c_void_p(q.data_ptr() + 4 * (i % 64)), _stream(stream)),
                    "xi_pass2_batched")


class GatherGraph:
    """The gathers of one wedge into the open blocks, captured once as a CUDA graph and replayed for every wedge
    while the same blocks are open: each block's launch reads the wedge's frames and rows from a device descriptor
    (xi_gather_step), which an upload rewrites before each replay. `key`: the open blocks the graph was captured
    for."""

    GRID = 148 * 8

    def __init__(self, key, grows_list, arenas, cnts, device="cuda"):
        self.key = key
        n = len(grows_list)
        self.size = C.sizeof(N.XiGatherStep)
        self.desc = torch.zeros(max(n, 1) * self.size, dtype=torch.uint8, device=device)
        self.graph = torch.cuda.CUDAGraph()
        self._keep = (grows_list, arenas, cnts)
        lib = N.load()
        base = self.desc.data_ptr()
        # captured on a side stream (nothing runs; no device-wide synchronisation, the allocator's cache is kept)
        cap = torch.cuda.Stream(device=self.desc.device)
        cap.wait_stream(torch.cuda.current_stream(self.desc.device))
        with torch.cuda.stream(cap):
            self.graph.capture_begin(capture_error_mode="thread_local")
            try:
                st = _stream(cap)
                for j, (g, a, c) in enumerate(zip(grows_list, arenas, cnts)):
                    N.check(lib.xi_gather_step(C.c_void_p(base + j * self.size), C.byref(g.s), N.ptr(a), N.ptr(c),
                                               self.GRID, st), "xi_gather_step")
            finally:
                self.graph.capture_end()

    def replay(self, steps):
        """steps: one XiGatherStep per block of the key, in order."""
        arr = (N.XiGatherStep * len(steps))(*steps)
        host = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8)
        if not _RING.upload(host, self.desc[:host.numel()], torch.cuda.current_stream(self.desc.device)):
            self.desc[:host.numel()].copy_(host.pin_memory(), non_blocking=True)
        with TIMER.span("gather", len(steps)):
            self.graph.replay()
