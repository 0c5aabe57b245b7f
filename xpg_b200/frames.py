"""Frame sources of the integration: how detector frames reach the device.

* `U32Frames`: raw uint32 frames (Eiger-style: 0xFFFFFFFF flagged, counts >= overload overloaded) in host memory
  (numpy, ideally pinned) or already on the device (torch). The kernels encode them (`xpg/io/images.py:72-102`).
  From a pinned torch tensor a transfer thread uploads them, mostly packed to one byte a pixel on the host's cores
  (`xi_pack_u8` / `xi_unpack_u8`).
* `BSLZ4Frames`: bitshuffle-LZ4 chunks (Eiger HDF5 chunks) of uint32 / uint16 counts: the LZ4 stage on the host's
  cores, the bit unshuffle on the device, then the uint32 path.
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


# transfers: a chunk goes raw when more than this fraction of its pixels need an exception pair
PACK_EXC_PER_PIXEL = 1.0 / 64
# raw chunks' worth of copies kept queued in the copy engine at most
QUEUED_CHUNKS = 3
# a second transfer thread copies chunks raw from the back of each wedge while the first packs from its front
RAW_THREAD = True


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


_STREAMS = {}


def _transfer_streams(device):
    """Streams of the transfer threads, one set per device for the whole process (the caching allocator reuses a
    stream's freed blocks only for that stream): raw copies, packed copies, and the unpacks (high priority, so that
    the widening of a chunk does not wait behind the integration's kernels)."""
    key = device.index
    if key not in _STREAMS:
        _STREAMS[key] = (torch.cuda.Stream(device=device), torch.cuda.Stream(device=device),
                         torch.cuda.Stream(device=device, priority=-1))
    return _STREAMS[key]


class _Job:
    """One wedge in transfer: chunks [lo, hi) are not yet taken; `left` are not yet issued."""

    def __init__(self, w, h, d, n_chunks):
        self.w, self.h, self.d = w, h, d
        self.lo, self.hi, self.left = 0, n_chunks, n_chunks


class _Feeder:
    """Transfers the wedges of a run from pinned host memory ahead of the integration, starting before the plan is
    made, in chunks of `chunk` frames; at most `depth` wedges are held on the device.

    Two threads share each wedge. The packing thread takes chunks from its front, packs each on the host's cores
    (xi_pack_u8: 1 byte a pixel plus exceptions) and uploads it, to be widened on the device (xi_unpack_u8); the raw
    thread takes chunks from its back and copies them as they are (4 bytes a pixel), keeping `queued` raw chunks'
    worth of copies waiting in the copy engine (it serves copies in submission order, across streams, so a small
    copy the integration issues meanwhile waits for little). Both stay busy until they meet, so the split between
    the link and the host's cores follows their speeds. Without packing one thread copies every chunk raw. The
    device frames are the same either way, bit for bit."""

    HOST_SLOTS = 8
    DEV_SLOTS = 6

    def __init__(self, host, first, wedges, oks, device, depth=4, chunk=2, queued=4, pack=True, raw_thread=True,
                 exc_per_pixel=PACK_EXC_PER_PIXEL, threads=0, stats=None):
        self.host, self.first = host, first
        self.wedges, self.oks = wedges, oks
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.s_raw, self.s_pk, self.s_un = _transfer_streams(self.device)
        self.ready = [threading.Event() for _ in wedges]
        self.out = [None] * len(wedges)
        self.held = [False] * len(wedges)   # the wedge took a slot
        self.slots = threading.Semaphore(depth)
        self.chunk, self.queued = chunk, queued
        self.pack, self.exc_per_pixel, self.threads = pack, exc_per_pixel, threads
        self.stats = stats if stats is not None else {}
        for k in ("h2d_bytes", "chunks_raw", "chunks_packed"):
            self.stats.setdefault(k, 0)
        self.cv = threading.Condition()
        self.jobs = []                      # wedges in transfer, in order
        self.owner_done = False
        self.pend = collections.deque()     # (copy event, raw chunks' worth of bytes), in submission order
        self.error = None
        self.stopping = False
        self.px_chunk = chunk * int(host.shape[1]) * int(host.shape[2])
        self.threads_ = [threading.Thread(target=self._guard, args=(self._owner,), daemon=True)]
        if pack and raw_thread:
            self.threads_.append(threading.Thread(target=self._guard, args=(self._raw_from_back,), daemon=True))
        for t in self.threads_:
            t.start()

    def _guard(self, fn):
        try:
            torch.cuda.set_device(self.device)
            fn()
        except BaseException as e:          # surfaced by get()
            with self.cv:
                self.error = self.error or e
                self.stopping = True
                self.cv.notify_all()
            for r in self.ready:
                r.set()

    # ---- the copy engine's queue
    def _backlog(self):
        with self.cv:
            while self.pend and self.pend[0][0].query():
                self.pend.popleft()
            return sum(u for _, u in self.pend)

    def _wait_backlog(self):
        while self._backlog() >= self.queued and not self.stopping:
            time.sleep(2e-4)                # polling lets the integration's thread run meanwhile

    # ---- one chunk
    def _raw(self, job, c):
        hc, dc = job.h[c * self.chunk:(c + 1) * self.chunk], job.d[c * self.chunk:(c + 1) * self.chunk]
        with torch.cuda.stream(self.s_raw):
            dc.copy_(hc, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.s_raw)
        with self.cv:
            self.pend.append((ev, hc.numel() / self.px_chunk))
            self.stats["h2d_bytes"] += 4 * hc.numel()
            self.stats["chunks_raw"] += 1

    def _packed(self, job, c, st):
        """Packs and uploads chunk c; False when it needs more exception pairs than a slot holds (send it raw)."""
        import ctypes as C
        from . import native
        hc, dc = job.h[c * self.chunk:(c + 1) * self.chunk], job.d[c * self.chunk:(c + 1) * self.chunk]
        if dc.data_ptr() % 16:
            return False
        n = hc.numel()
        hk, hbuf = _HOST_SLOTS.take(st["slot_bytes"], self.HOST_SLOTS)
        hp = hbuf.data_ptr()
        rc = st["lib"].xi_pack_u8(C.c_void_p(hc.data_ptr()), n, C.c_void_p(hp), C.c_void_p(hp + st["plane"]),
                                  st["cap"], self.threads, C.byref(st["n_exc"]))
        if rc == native.XI_E_LIMIT:
            return False
        native.check(rc, "xi_pack_u8")
        ne = st["n_exc"].value
        nbytes = st["plane"] + 8 * ne
        dk = st["dk"]
        st["dk"] = (dk + 1) % self.DEV_SLOTS
        dbuf = st["dev"][dk]
        if st["dev_ev"][dk] is not None:
            self.s_pk.wait_event(st["dev_ev"][dk])      # its last unpack has read it
        with torch.cuda.stream(self.s_pk):
            dbuf[:nbytes].copy_(hbuf[:nbytes], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.s_pk)
        _HOST_SLOTS.events[hk] = ev
        self.s_un.wait_event(ev)
        dp = dbuf.data_ptr()
        native.check(st["lib"].xi_unpack_u8(C.c_void_p(dp), n, C.c_void_p(dp + st["plane"]), ne,
                                            C.c_void_p(dc.data_ptr()), C.c_void_p(self.s_un.cuda_stream)),
                     "xi_unpack_u8")
        ue = torch.cuda.Event()
        ue.record(self.s_un)
        st["dev_ev"][dk] = ue
        with self.cv:
            self.pend.append((ev, nbytes / (4.0 * self.px_chunk)))
            self.stats["h2d_bytes"] += nbytes
            self.stats["chunks_packed"] += 1
        return True

    def _issued(self, job):
        """One chunk of the job issued; after its last one the wedge's ready event follows every copy and unpack."""
        with self.cv:
            job.left -= 1
            if job.left:
                return
            ev = torch.cuda.Event()
            ev.record(self.s_raw)
            self.s_un.wait_event(ev)
            ready = torch.cuda.Event()
            ready.record(self.s_un)
            self.out[job.w] = (job.d, ready)
            self.ready[job.w].set()

    def _take(self, job, front):
        with self.cv:
            if job.lo >= job.hi:
                return None
            if front:
                job.lo += 1
                return job.lo - 1
            job.hi -= 1
            return job.hi

    # ---- the threads
    def _owner(self):
        """Opens the wedges in order and works on each from its front (packing, or raw copies without packing)."""
        st = None
        if self.pack:
            import ctypes as C
            from . import native
            plane = (self.px_chunk + 15) // 16 * 16
            cap = max(1024, int(self.px_chunk * self.exc_per_pixel))
            st = {"lib": native.load(), "plane": plane, "cap": cap, "slot_bytes": plane + 8 * cap,
                  "n_exc": C.c_int64(), "dk": 0, "dev_ev": [None] * self.DEV_SLOTS}
            with torch.cuda.stream(self.s_pk):
                st["dev"] = [torch.empty(plane + 8 * cap, dtype=torch.uint8, device=self.device)
                             for _ in range(self.DEV_SLOTS)]
            for t in st["dev"]:
                t.record_stream(self.s_un)
        try:
            for w, (fa, fb) in enumerate(self.wedges):
                if not self.oks[w].any():
                    self.ready[w].set()
                    continue
                self.slots.acquire()
                if self.stopping:
                    break
                self.held[w] = True
                h = self.host[fa - self.first:fb - self.first + 1]
                with torch.cuda.stream(self.s_raw):
                    d = torch.empty(h.shape, dtype=h.dtype, device=self.device)
                d.record_stream(self.s_un)       # unpacks write it from their own stream
                job = _Job(w, h, d, (h.shape[0] + self.chunk - 1) // self.chunk)
                with self.cv:
                    self.jobs.append(job)
                    self.cv.notify_all()
                while not self.stopping:
                    c = self._take(job, True)
                    if c is None:
                        break
                    if not (self.pack and self._packed(job, c, st)):
                        if not self.pack:
                            self._wait_backlog()
                        self._raw(job, c)
                    self._issued(job)
        finally:
            with self.cv:
                self.owner_done = True
                self.cv.notify_all()

    def _raw_from_back(self):
        """Raw copies from the back of the earliest wedge with chunks left, while the copy engine has room."""
        k = 0
        while True:
            with self.cv:
                while k >= len(self.jobs) and not self.owner_done and not self.stopping:
                    self.cv.wait(0.05)
                if self.stopping or k >= len(self.jobs):
                    return
                job = self.jobs[k]
            self._wait_backlog()
            c = self._take(job, False)
            if c is None:
                k += 1
                continue
            self._raw(job, c)
            self._issued(job)

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
        with self.cv:
            self.stopping = True
            self.cv.notify_all()
        for _ in range(len(self.wedges) + 1):
            self.slots.release()
        for t in self.threads_:
            t.join()


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
        return _Feeder(h, self.first, wedges, oks, self.device, depth=self._depth(wedges), queued=QUEUED_CHUNKS,
                       pack=self.pack, raw_thread=RAW_THREAD, exc_per_pixel=PACK_EXC_PER_PIXEL, stats=self.transfer)

    def _depth(self, wedges):
        """Wedges the transfer may hold on the device at once: as many as half the free device memory takes (at
        least 4), so that the transfer runs ahead of an integration that is still planning."""
        dev = torch.device(self.device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        free = torch.cuda.mem_get_info(dev)[0] + torch.cuda.memory_reserved(dev) - torch.cuda.memory_allocated(dev)
        per = max(fb - fa + 1 for fa, fb in wedges) * self.ny * self.nx * 4 if wedges else 1
        return max(4, min(len(wedges), int(0.5 * free // per)))

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


class BSLZ4Frames:
    """Frames as bitshuffle-LZ4 chunks (HDF5 filter 32008: Eiger data read with the filter bypassed, as XPG's
    `read_chunk` gives them, `xpg/io/images.py:384-396`) of uint32 or uint16 counts. Each wedge: the LZ4 stage of its
    chunks on the host's cores (xi_bslz4_lz4_stage) into pinned staging, one upload, the bit unshuffle on the device
    (xi_bitunshuffle) into uint32 frames; from there the uint32 path (the gather encodes the counts: all-ones flagged,
    counts >= overload overloaded), so the results are those of the same frames given raw.

    chunks: a sequence (frame `first + i` at index i) or a callable frame -> chunk bytes."""

    def __init__(self, chunks, ny, nx, esize=4, first=1, last=None, overload=1 << 20, min_valid=0, device="cuda"):
        if esize not in (2, 4):
            raise ValueError("esize: 2 or 4 bytes")
        self.chunks = chunks
        self.first = int(first)
        self.last = int(last) if last is not None else self.first + len(chunks) - 1
        self.ny, self.nx, self.esize = int(ny), int(nx), int(esize)
        self.overload = int(overload) if overload is not None else None
        self.min_valid = int(min_valid)
        self.device = device
        self.resident = False
        self._ring = _PinnedRing(torch.uint8)

    def _chunk(self, f):
        c = self.chunks(f) if callable(self.chunks) else self.chunks[f - self.first]
        if c is None:
            raise RuntimeError(f"frame {f}: no chunk")
        return np.frombuffer(c, np.uint8) if not isinstance(c, np.ndarray) else np.ascontiguousarray(c, np.uint8)

    def wedge(self, f_a, f_b, ok=None, stream=None):
        import ctypes as C
        from . import native
        lib = native.load()
        n = f_b - f_a + 1
        nel = self.ny * self.nx
        fb = nel * self.esize
        k, buf = self._ring.take(n * fb)
        base = buf.data_ptr()
        nb, be = C.c_int64(), C.c_int64()
        belem = [0] * n
        for w in range(n):
            if ok is not None and not ok[w]:
                continue                                   # excluded: never read (the gather skips the frame)
            c = self._chunk(f_a + w)
            native.check(lib.xi_bslz4_lz4_stage(c.ctypes.data, c.size, self.esize, C.c_void_p(base + w * fb), fb,
                                                0, C.byref(nb), C.byref(be)), f"frame {f_a + w}: xi_bslz4_lz4_stage")
            if nb.value != fb:
                raise RuntimeError(f"frame {f_a + w}: chunk of {nb.value} bytes, frame of {fb}")
            belem[w] = be.value
        dev = self._ring.upload(k, buf, self.device)
        d = torch.empty((n, self.ny, self.nx), dtype=torch.int32, device=dev.device)
        st = native.stream_handle()
        for w in range(n):
            if belem[w]:
                native.check(lib.xi_bitunshuffle(C.c_void_p(dev.data_ptr() + w * fb), nel, self.esize, belem[w],
                                                 C.c_void_p(d[w].data_ptr()), st), "xi_bitunshuffle")
        return d, False


class PackedStore:
    """uint32 frames held in the library's transfer encoding (`xi_pack_u8`: one byte a pixel, exception pairs for
    counts of 254 and above): about a quarter of the raw frames' size, so a whole sweep fits in host memory or in
    HBM. Frames live in segments (uint8 tensors, pinned host memory or device memory) at 16-byte aligned offsets;
    a frame with more than 1/64 exception pixels is kept raw (4 bytes a pixel). `to(device)` copies the segments to
    the device (frames resident in HBM in packed form)."""

    SEGMENT = 1 << 31

    def __init__(self, n_frames, ny, nx, segments=None, index=None):
        self.n_frames, self.ny, self.nx = int(n_frames), int(ny), int(nx)
        self.P = self.ny * self.nx
        self.plane = (self.P + 15) // 16 * 16
        self.segments = segments if segments is not None else []
        self.index = index if index is not None else np.zeros((self.n_frames, 4), np.int64)   # seg, off, n_exc, raw
        self._fill = 0

    @property
    def nbytes(self):
        return int(sum(int(self.frame_bytes(k)) for k in range(self.n_frames)))

    def frame_bytes(self, k):
        seg, off, ne, raw = self.index[k]
        return 4 * self.P if raw else self.plane + (8 * ne + 15) // 16 * 16

    def _room(self, nbytes):
        if not self.segments or self._fill + nbytes > self.segments[-1].numel():
            self.segments.append(torch.empty(max(self.SEGMENT, nbytes), dtype=torch.uint8, pin_memory=True))
            self._fill = 0
        off = self._fill
        self._fill += (nbytes + 15) // 16 * 16
        return len(self.segments) - 1, off

    def add_wedge(self, first_k, host_u32, threads=0):
        """Packs frames first_k.. from a pinned uint32 host tensor (n, ny, nx) on the host's cores."""
        import ctypes as C
        from . import native
        lib = native.load()
        cap = max(1024, self.P // 64)
        n_exc = C.c_int64()
        for w in range(int(host_u32.shape[0])):
            src = host_u32[w]
            seg, off = self._room(self.plane + 8 * cap)
            base = self.segments[seg].data_ptr() + off
            rc = lib.xi_pack_u8(C.c_void_p(src.data_ptr()), self.P, C.c_void_p(base), C.c_void_p(base + self.plane),
                                cap, threads, C.byref(n_exc))
            if rc == native.XI_E_LIMIT:                  # too many exceptions: the frame stays raw
                self._fill = off
                seg, off = self._room(4 * self.P)
                self.segments[seg][off:off + 4 * self.P].copy_(src.reshape(-1).view(torch.uint8))
                self.index[first_k + w] = (seg, off, 0, 1)
                continue
            native.check(rc, "xi_pack_u8")
            used = self.plane + (8 * n_exc.value + 15) // 16 * 16
            self._fill = off + used
            self.index[first_k + w] = (seg, off, n_exc.value, 0)

    def to(self, device):
        """The same frames with every segment copied to `device` (trimmed to what the frames use)."""
        used = np.zeros(len(self.segments), np.int64)
        for k in range(self.n_frames):
            seg, off = int(self.index[k, 0]), int(self.index[k, 1])
            used[seg] = max(used[seg], off + self.frame_bytes(k))
        segs = [s[:int(u)].to(device) for s, u in zip(self.segments, used)]
        return PackedStore(self.n_frames, self.ny, self.nx, segs, self.index.copy())

    def unpack_frames(self, k0, n, out, stream, ok=None):
        """Frames k0..k0+n-1 into out (device int32 (n, ny, nx), 16-byte aligned) with one launch on `stream`; the
        store must be on the device; frames with ok False are skipped (left as they are)."""
        import ctypes as C
        from . import native
        from .device import TIMER, h2d
        arr = (native.XiPackedFrame * n)()
        m = 0
        order = []
        for i in range(n):
            if ok is not None and not ok[i]:
                continue
            seg, off, ne, raw = (int(v) for v in self.index[k0 + i])
            base = self.segments[seg].data_ptr() + off
            arr[m].plane, arr[m].exc, arr[m].n_exc, arr[m].raw = base, base + self.plane, ne, raw
            order.append(i)
            m += 1
        if m == 0:
            return
        if m != n:                              # excluded frames: one launch per run of kept frames
            for i in range(m):
                self.unpack(k0 + order[i], out[order[i]], stream)
            return
        d = h2d(np.frombuffer(bytes(arr), np.uint8), None, out.device)
        with TIMER.span("unpack"):
            native.check(native.load().xi_unpack_u8_frames(C.c_void_p(d.data_ptr()), n, self.P,
                                                            C.c_void_p(out.data_ptr()), self.P,
                                                            C.c_void_p(stream.cuda_stream)), "xi_unpack_u8_frames")

    def unpack(self, k, out, stream):
        """Frame k into out (device uint32 / int32 frame, 16-byte aligned) on `stream`; the store must be on the
        device."""
        import ctypes as C
        from . import native
        seg, off, ne, raw = (int(v) for v in self.index[k])
        src = self.segments[seg]
        if raw:
            with torch.cuda.stream(stream):
                out.reshape(-1).view(torch.uint8).copy_(src[off:off + 4 * self.P], non_blocking=True)
            return
        base = src.data_ptr() + off
        native.check(native.load().xi_unpack_u8(C.c_void_p(base), self.P, C.c_void_p(base + self.plane), ne,
                                                C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream)),
                     "xi_unpack_u8")


def pack_generated(render, n_frames, ny, nx, wedge=16, device="cuda"):
    """PackedStore of n_frames frames rendered on the device: `render(first_k, n, out)` writes frames
    first_k..first_k+n-1 (0-based) into the device int32 tensor out (n, ny, nx); each wedge is read back into pinned
    memory and packed on the host's cores."""
    store = PackedStore(n_frames, ny, nx)
    dev = torch.empty((wedge, ny, nx), dtype=torch.int32, device=device)
    host = torch.empty((wedge, ny, nx), dtype=torch.int32, pin_memory=True)
    for k in range(0, n_frames, wedge):
        n = min(wedge, n_frames - k)
        render(k, n, dev[:n])
        host[:n].copy_(dev[:n])
        store.add_wedge(k, host[:n])
    return store


class _PackedFeeder:
    """Unpacks the wedges of a run from a PackedStore ahead of the integration: one thread issues, per wedge, the
    packed frames' copies to the device (from pinned host memory, on a copy stream; none when the store is on the
    device) and their unpacks (on a stream of their own); at most `depth` wedges are held on the device."""

    def __init__(self, store, first, wedges, oks, device, depth=3, stats=None):
        self.store, self.first = store, first
        self.wedges, self.oks = wedges, oks
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.s_cp, _, self.s_un = _transfer_streams(self.device)
        self.on_device = store.segments[0].is_cuda if store.segments else True
        self.ready = [threading.Event() for _ in wedges]
        self.out = [None] * len(wedges)
        self.held = [False] * len(wedges)
        self.slots = threading.Semaphore(depth)
        self.stats = stats if stats is not None else {}
        self.stats.setdefault("h2d_bytes", 0)
        self.error = None
        self.stopping = False
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        from .device import TIMER
        try:
            torch.cuda.set_device(self.device)
            st = self.store
            stage, stage_ev = [], []
            if not self.on_device:
                cap = max(st.frame_bytes(k) for k in range(st.n_frames)) if st.n_frames else 16
                with torch.cuda.stream(self.s_cp):
                    stage = [torch.empty(cap, dtype=torch.uint8, device=self.device) for _ in range(4)]
                stage_ev = [None] * len(stage)
                for t in stage:
                    t.record_stream(self.s_un)
            q = 0
            for w, (fa, fb) in enumerate(self.wedges):
                if not self.oks[w].any():
                    self.ready[w].set()
                    continue
                self.slots.acquire()
                if self.stopping:
                    return
                self.held[w] = True
                n = fb - fa + 1
                with torch.cuda.stream(self.s_un):
                    d = torch.empty((n, st.ny, st.nx), dtype=torch.int32, device=self.device)
                for i in range(n):
                    if not self.oks[w][i]:
                        continue
                    k = fa - self.first + i
                    if self.on_device:
                        with torch.cuda.stream(self.s_un), TIMER.span("unpack"):
                            st.unpack(k, d[i], self.s_un)
                        continue
                    seg, off = int(st.index[k, 0]), int(st.index[k, 1])
                    nb = st.frame_bytes(k)
                    if stage_ev[q] is not None:
                        self.s_cp.wait_event(stage_ev[q])       # the unpack that last read this slot has run
                    with torch.cuda.stream(self.s_cp):
                        stage[q][:nb].copy_(st.segments[seg][off:off + nb], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(self.s_cp)
                    self.s_un.wait_event(ev)
                    one = PackedStore(1, st.ny, st.nx, [stage[q]], np.array([[0, 0] + list(st.index[k, 2:])]))
                    with torch.cuda.stream(self.s_un), TIMER.span("unpack"):
                        one.unpack(0, d[i], self.s_un)
                    ue = torch.cuda.Event()
                    ue.record(self.s_un)
                    stage_ev[q] = ue
                    q = (q + 1) % len(stage)
                    self.stats["h2d_bytes"] += nb
                ready = torch.cuda.Event()
                ready.record(self.s_un)
                self.out[w] = (d, ready)
                self.ready[w].set()
        except BaseException as e:
            self.error = e
            for r in self.ready:
                r.set()

    def get(self, w):
        self.ready[w].wait()
        if self.error is not None:
            raise RuntimeError("packed frame transfer failed") from self.error
        d, ev = self.out[w]
        self.out[w] = None
        cur = torch.cuda.current_stream()
        cur.wait_event(ev)
        d.record_stream(cur)
        return d

    def done_with(self, w):
        self.ready[w].wait()
        self.out[w] = None
        if self.held[w]:
            self.held[w] = False
            self.slots.release()

    def close(self):
        self.stopping = True
        for _ in range(len(self.wedges) + 1):
            self.slots.release()
        self.t.join()


class PackedFrames:
    """Raw uint32 frames given as a PackedStore (in pinned host memory: each wedge's packed bytes cross the link and
    are widened on the device; in device memory: widened there), then the uint32 path: the same results as the
    frames given raw."""

    def __init__(self, store, first=1, overload=1 << 20, min_valid=0, device="cuda", depth=3):
        self.store = store
        self.first = int(first)
        self.last = self.first + store.n_frames - 1
        self.ny, self.nx = store.ny, store.nx
        self.overload = int(overload) if overload is not None else None
        self.min_valid = int(min_valid)
        self.device = device
        self.resident = False
        self.depth = depth
        self.transfer = {}
        self._buf = None

    @property
    def on_device(self):
        return bool(self.store.segments) and self.store.segments[0].is_cuda

    @property
    def hide_transfer(self):
        return not self.on_device

    def feeder(self, wedges, oks):
        """A transfer thread when the store is in host memory; None when it is in HBM (wedges widened in place)."""
        if self.on_device:
            return None
        return _PackedFeeder(self.store, self.first, wedges, oks, self.device, self.depth, self.transfer)

    def wedge(self, f_a, f_b, ok=None, stream=None):
        """Frames f_a..f_b widened into the source's wedge buffer (reused wedge after wedge: the next wedge's unpack
        is queued on the stream after the kernels that read this one)."""
        from .device import POOL
        n = f_b - f_a + 1
        if self._buf is None or self._buf.numel() < n * self.ny * self.nx:
            POOL.give(self._buf)
            self._buf = POOL.take(n * self.ny * self.nx, torch.int32, self.device)
        d = self._buf[:n * self.ny * self.nx].view(n, self.ny, self.nx)
        st = stream if stream is not None else torch.cuda.current_stream()
        self.store.unpack_frames(f_a - self.first, n, d, st, ok)
        return d, False


class GeneratedFrames:
    """Frames of a synthetic sweep rendered on the device as the integration asks for them (the generator of
    xpg_b200.synth, `DeviceSpots`): each wedge is rendered into a fresh device buffer on the current stream, then the
    uint32 path. For sweeps and request streams whose frames are produced on the device (nothing crosses the host
    link); the rendering is part of the timed work."""

    def __init__(self, spots, first=1, last=None, overload=1 << 20, device="cuda"):
        spec = spots.spec
        self.spots = spots
        self.first = int(first)
        self.last = int(last) if last is not None else spec.nframes
        self.ny, self.nx = spec.ny, spec.nx
        self.overload = int(overload) if overload is not None else None
        self.min_valid = 0
        self.device = device
        self.resident = False
        self.hide_transfer = False
        self._buf = None

    def wedge(self, f_a, f_b, ok=None, stream=None):
        """Frames f_a..f_b rendered into the source's wedge buffer (reused wedge after wedge, in stream order)."""
        from .device import POOL, TIMER
        n = f_b - f_a + 1
        if self._buf is None or self._buf.numel() < n * self.ny * self.nx:
            POOL.give(self._buf)
            self._buf = POOL.take(n * self.ny * self.nx, torch.int32, self.device)
        d = self._buf[:n * self.ny * self.nx].view(n, self.ny, self.nx)
        with TIMER.span("generate", 2):
            self.spots.render(f_a, f_b - f_a + 1, d, stream)
        return d, False


def as_frame_source(images, device="cuda"):
    if isinstance(images, (U32Frames, ImageSetFrames, BSLZ4Frames, PackedFrames, GeneratedFrames)):
        return images
    if _bitshuffled_imageset(images):
        return BSLZ4Frames(images.read_chunk, images.ny, images.nx, esize=int(np.dtype(images.dtype).itemsize),
                           first=images.first, last=images.last, overload=getattr(images, "overload", None),
                           min_valid=getattr(images, "min_valid", 0), device=device)
    if hasattr(images, "get") and hasattr(images, "first"):
        return ImageSetFrames(images, device)
    raise TypeError("images: a U32Frames, ImageSetFrames or an XPG-style ImageSet (first, last, nx, ny, get)")


def _bitshuffled_imageset(images):
    """An XPG image set whose frames are plain bitshuffle-LZ4 chunks the device can finish (`bitshuffled_ok`,
    `xpg/io/images.py:157-160`, `:365-382`) and whose encoding is the uint32 path's: no static pixel mask (a masked
    pixel there reads -1 even when overloaded), no offset or dark frame."""
    try:
        if not (hasattr(images, "read_chunk") and images.bitshuffled_ok()):
            return False
    except Exception:
        return False
    sm = getattr(images, "static_mask", None)
    return sm is None or bool(np.asarray(sm).all())
