"""Frame sources of the integration: how detector frames reach the device.

* `U32Frames`: raw uint32 frames (Eiger-style: 0xFFFFFFFF flagged, counts >= overload overloaded) in host memory
  (numpy, ideally pinned) or already on the device (torch). The kernels encode them (`xpg/io/images.py:72-102`).
  From a pinned torch tensor a transfer thread uploads them, mostly packed to one byte a pixel on the host's cores
  (`xi_pack_u8` / `xi_unpack_u8`).
* `ImageSetFrames`: any XPG-style image set (`first`, `last`, `nx`, `ny`, `get(frame)` -> float32 frame with -1
  masked / -2 overloaded, `xpg/io/images.py:59-102`); frames are stacked per wedge on the host and uploaded as
  float32.

A wedge is a run of consecutive frame numbers; `wedge(f_a, f_b, ok)` returns the device tensor (n, ny, nx) of frames
f_a..f_b (1-based, inclusive) and the XiFrames encoding parameters. Frames whose `ok` flag is False (excluded) are
neither read nor uploaded.
"""
from __future__ import annotations

import collections
import threading
import time

import numpy as np
import torch


# transfer thread: a chunk is packed while at least this many raw chunks' worth of copies are queued ...
PACK_MIN_BACKLOG = 1.0
# ... and goes raw when more than this fraction of its pixels need an exception pair
PACK_EXC_PER_PIXEL = 1.0 / 64
# raw chunks' worth of copies the transfer thread keeps queued at most
QUEUED_CHUNKS = 4


class _Uploads:
    """Wedge transfers on a copy stream of their own: a wedge's upload overlaps the kernels of the wedges before it.
    The compute stream waits for each wedge's copy before its gathers; at most `depth` wedges are in flight (device
    memory)."""

    def __init__(self, depth=4):
        self.stream = None
        self.inflight = []
        self.depth = depth

    def upload(self, h, device):
        cur = torch.cuda.current_stream()
        if self.stream is None:
            self.stream = torch.cuda.Stream()
        while len(self.inflight) >= self.depth:
            self.inflight.pop(0).synchronize()
        with torch.cuda.stream(self.stream):
            d = h.to(device, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        cur.wait_event(ev)
        d.record_stream(cur)                 # the compute stream reads it: no reuse before its kernels ran
        self.inflight.append(ev)
        return d, ev


_UPLOADS = _Uploads()


class _HostSlots:
    """Pinned staging buffers of packed chunks, kept across runs (pinning memory is slow); a slot is rewritten only
    after the copy that read it finished."""

    def __init__(self):
        self.nbytes = 0
        self.bufs, self.events = [], []
        self.k = 0
        self.lock = threading.Lock()

    def take(self, nbytes, n_slots):
        with self.lock:
            return self._take(nbytes, n_slots)

    def _take(self, nbytes, n_slots):
        if nbytes > self.nbytes or len(self.bufs) != n_slots:
            self.nbytes = max(nbytes, self.nbytes)
            self.bufs = [torch.empty(self.nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(n_slots)]
            self.events = [None] * n_slots
            self.k = 0
        k = self.k
        self.k = (k + 1) % n_slots
        ev = self.events[k]
        if ev is not None:
            while not ev.query():
                time.sleep(2e-4)
            self.events[k] = None
        return k, self.bufs[k]


_HOST_SLOTS = _HostSlots()


class _Feeder:
    """Transfers the wedges of a run from pinned host memory ahead of the integration, from a thread of its own,
    starting before the plan is made, in copies of `chunk` frames on a copy stream (the copy engine serves copies in
    submission order, across streams, so at most `queued` raw chunks' worth of bytes wait in it and a small copy the
    integration issues meanwhile waits for little); at most `depth` wedges are held on the device.

    A chunk goes raw (4 bytes a pixel) or packed by xi_pack_u8 on the host's cores (1 byte a pixel plus exceptions,
    widened back on the device by xi_unpack_u8 on a second stream). The thread packs the next chunk while at least
    `min_backlog` raw chunks' worth of copies are queued, and sends it raw otherwise, so that the link never waits
    for the packing: the split adapts to the link's and the host's speeds. The device frames are the same either way,
    bit for bit."""

    HOST_SLOTS = 8
    DEV_SLOTS = 3

    def __init__(self, host, first, wedges, oks, device, depth=4, chunk=2, queued=4, pack=True,
                 min_backlog=PACK_MIN_BACKLOG, exc_per_pixel=PACK_EXC_PER_PIXEL, threads=0, stats=None):
        self.host, self.first = host, first
        self.wedges, self.oks = wedges, oks
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(device=self.device)
        self.unpack_stream = torch.cuda.Stream(device=self.device) if pack else None
        self.ready = [threading.Event() for _ in wedges]
        self.out = [None] * len(wedges)
        self.held = [False] * len(wedges)   # the wedge took a slot
        self.slots = threading.Semaphore(depth)
        self.chunk, self.queued = chunk, queued
        self.pack, self.min_backlog = pack, min_backlog
        self.exc_per_pixel, self.threads = exc_per_pixel, threads
        self.stats = stats if stats is not None else {}
        for k in ("h2d_bytes", "chunks_raw", "chunks_packed"):
            self.stats.setdefault(k, 0)
        self.error = None
        self.stopping = False
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        try:
            torch.cuda.set_device(self.device)
            self._transfer()
        except BaseException as e:          # surfaced by get()
            self.error = e
            for r in self.ready:
                r.set()

    def _transfer(self):
        import ctypes as C
        from . import native
        lib = native.load() if self.pack else None
        s1, s2 = self.stream, self.unpack_stream
        ny, nx = int(self.host.shape[1]), int(self.host.shape[2])
        px_chunk = self.chunk * ny * nx
        plane_bytes = (px_chunk + 15) // 16 * 16
        cap = max(1024, int(px_chunk * self.exc_per_pixel))
        slot_bytes = plane_bytes + 8 * cap
        dev_slots, dev_events = [], []
        if self.pack:
            with torch.cuda.stream(s1):
                dev_slots = [torch.empty(slot_bytes, dtype=torch.uint8, device=self.device)
                             for _ in range(self.DEV_SLOTS)]
            for t in dev_slots:
                t.record_stream(s2)
            dev_events = [None] * self.DEV_SLOTS
        dk = 0
        n_exc = C.c_int64() if self.pack else None
        pend = collections.deque()            # (copy event on s1, raw chunks' worth of bytes)

        def backlog():
            while pend and pend[0][0].query():
                pend.popleft()
            return sum(u for _, u in pend)

        for w, (fa, fb) in enumerate(self.wedges):
            if not self.oks[w].any():
                self.ready[w].set()
                continue
            self.slots.acquire()
            if self.stopping:
                break
            self.held[w] = True
            h = self.host[fa - self.first:fb - self.first + 1]
            with torch.cuda.stream(s1):
                d = torch.empty(h.shape, dtype=h.dtype, device=self.device)
            if self.pack:
                d.record_stream(s2)              # unpacks write it from the second stream
            last = None
            for c0 in range(0, h.shape[0], self.chunk):
                hc, dc = h[c0:c0 + self.chunk], d[c0:c0 + self.chunk]
                n = hc.numel()
                units = n / px_chunk
                q = backlog()
                while q >= self.queued:
                    time.sleep(2e-4)            # polling lets the integration's thread run meanwhile
                    q = backlog()
                packed = False
                if self.pack and q >= self.min_backlog and dc.data_ptr() % 16 == 0:
                    hk, hbuf = _HOST_SLOTS.take(slot_bytes, self.HOST_SLOTS)
                    hp = hbuf.data_ptr()
                    rc = lib.xi_pack_u8(C.c_void_p(hc.data_ptr()), n, C.c_void_p(hp),
                                        C.c_void_p(hp + plane_bytes), cap, self.threads, C.byref(n_exc))
                    if rc == native.XI_OK:
                        packed = True
                    elif rc != native.XI_E_LIMIT:   # too many exceptions: this chunk goes raw
                        native.check(rc, "xi_pack_u8")
                if packed:
                    ne = n_exc.value
                    nbytes = plane_bytes + 8 * ne
                    dbuf = dev_slots[dk]
                    if dev_events[dk] is not None:
                        s1.wait_event(dev_events[dk])   # its last unpack has read it
                    with torch.cuda.stream(s1):
                        dbuf[:nbytes].copy_(hbuf[:nbytes], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(s1)
                    _HOST_SLOTS.events[hk] = ev
                    s2.wait_event(ev)
                    dp = dbuf.data_ptr()
                    native.check(lib.xi_unpack_u8(C.c_void_p(dp), n, C.c_void_p(dp + plane_bytes), ne,
                                                  C.c_void_p(dc.data_ptr()), C.c_void_p(s2.cuda_stream)),
                                 "xi_unpack_u8")
                    ue = torch.cuda.Event()
                    ue.record(s2)
                    dev_events[dk] = ue
                    dk = (dk + 1) % self.DEV_SLOTS
                    pend.append((ev, nbytes / (4.0 * px_chunk)))
                    self.stats["h2d_bytes"] += nbytes
                    self.stats["chunks_packed"] += 1
                else:
                    with torch.cuda.stream(s1):
                        dc.copy_(hc, non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(s1)
                    pend.append((ev, units))
                    self.stats["h2d_bytes"] += 4 * n
                    self.stats["chunks_raw"] += 1
                last = ev
            if self.pack:                        # the wedge is ready when its raw copies and its unpacks are done
                s2.wait_event(last)
                last = torch.cuda.Event()
                last.record(s2)
            self.out[w] = (d, last)
            self.ready[w].set()

    def get(self, w):
        """Wedge w on the device, ordered before the current stream's next work."""
        self.ready[w].wait()
        if self.error is not None:
            raise RuntimeError("frame transfer failed") from self.error
        d, ev = self.out[w]
        self.out[w] = None
        cur = torch.cuda.current_stream()
        cur.wait_event(ev)
        d.record_stream(cur)                 # no reuse of its memory before the current stream's kernels ran
        return d

    def done_with(self, w):
        """The wedge's kernels are queued (or it was not needed): its slot may take the next wedge."""
        self.ready[w].wait()
        self.out[w] = None
        if self.held[w]:
            self.held[w] = False
            self.slots.release()

    def close(self):
        self.stopping = True
        for _ in range(len(self.wedges) + 1):
            self.slots.release()
        self.thread.join()


class _PinnedRing:
    """Two pinned staging buffers used alternately; a buffer is refilled only after its last upload finished."""

    def __init__(self, dtype):
        self.dtype = dtype
        self.bufs = [None, None]
        self.events = [None, None]
        self.k = 0

    def take(self, n):
        k = self.k
        self.k ^= 1
        if self.events[k] is not None:
            self.events[k].synchronize()
            self.events[k] = None
        if self.bufs[k] is None or self.bufs[k].numel() < n:
            self.bufs[k] = torch.empty(n, dtype=self.dtype, pin_memory=True)
        return k, self.bufs[k][:n]

    def upload(self, k, h, device):
        d, ev = _UPLOADS.upload(h, device)
        self.events[k] = ev
        return d


class U32Frames:
    def __init__(self, data, first=1, overload=1 << 20, min_valid=0, device="cuda", pack=True):
        self.data = data
        self.first = int(first)
        n = int(data.shape[0])
        self.last = self.first + n - 1
        self.ny, self.nx = int(data.shape[1]), int(data.shape[2])
        self.overload = int(overload) if overload is not None else None
        self.min_valid = int(min_valid)
        self.device = device
        self.on_device = torch.is_tensor(data) and data.is_cuda
        self.resident = self.on_device          # frames already in device memory: nothing to transfer
        self.pack = pack                        # packed transfers (xi_pack_u8) from a pinned tensor
        self.transfer = {}                      # the transfer thread's counts: h2d_bytes, chunks_raw, chunks_packed
        self._ring = _PinnedRing(torch.int32)

    def _host_slice(self, a, b):
        return self.data[a - self.first:b - self.first + 1]

    def feeder(self, wedges, oks):
        """A transfer thread for the run's wedges when the frames are a pinned host tensor (None otherwise)."""
        d = self.data
        if self.on_device or not torch.is_tensor(d) or not d.is_pinned():
            return None
        h = d if d.dtype == torch.int32 else d.view(torch.int32)
        return _Feeder(h, self.first, wedges, oks, self.device, queued=QUEUED_CHUNKS, pack=self.pack,
                       min_backlog=PACK_MIN_BACKLOG, exc_per_pixel=PACK_EXC_PER_PIXEL, stats=self.transfer)

    def wedge(self, f_a, f_b, ok=None, stream=None):
        if self.on_device:
            t = self.data[f_a - self.first:f_b - self.first + 1]
            return (t if t.dtype in (torch.int32, torch.float32) else t.view(torch.int32)), False
        src = self._host_slice(f_a, f_b)
        if torch.is_tensor(src):
            h = src if src.dtype == torch.int32 else src.view(torch.int32)
            if not h.is_pinned():
                return h.to(self.device), False
            return _UPLOADS.upload(h, self.device)[0], False
        n = src.shape[0]
        k, buf = self._ring.take(n * self.ny * self.nx)
        h = buf.view(n, self.ny, self.nx)
        np.copyto(h.numpy(), np.ascontiguousarray(src).view(np.int32))
        return self._ring.upload(k, h, self.device), False


class ImageSetFrames:
    """Adapter of an XPG ImageSet: frames arrive already encoded as float32."""

    def __init__(self, images, device="cuda"):
        self.images = images
        self.first, self.last = int(images.first), int(images.last)
        self.ny, self.nx = int(images.ny), int(images.nx)
        self.overload = None
        self.min_valid = 0
        self.device = device
        self.resident = False
        self._ring = _PinnedRing(torch.float32)

    def wedge(self, f_a, f_b, ok=None, stream=None):
        n = f_b - f_a + 1
        k, buf = self._ring.take(n * self.ny * self.nx)
        h = buf.view(n, self.ny, self.nx)
        hn = h.numpy()
        for w in range(n):
            if ok is not None and not ok[w]:
                hn[w] = -1.0
                continue
            hn[w] = self.images.get(f_a + w)
        return self._ring.upload(k, h, self.device), True


def as_frame_source(images, device="cuda"):
    if isinstance(images, (U32Frames, ImageSetFrames)):
        return images
    if hasattr(images, "get") and hasattr(images, "first"):
        return ImageSetFrames(images, device)
    raise TypeError("images: a U32Frames, ImageSetFrames or an XPG-style ImageSet (first, last, nx, ny, get)")
