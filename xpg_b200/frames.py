"""Frame sources of the integration: how detector frames reach the device.

* `U32Frames`: raw uint32 frames (Eiger-style: 0xFFFFFFFF flagged, counts >= overload overloaded) in host memory
  (numpy, ideally pinned) or already on the device (torch). The kernels encode them (`xpg/io/images.py:72-102`).
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


class _Feeder:
    """Transfers the wedges of a run from pinned host memory ahead of the integration, from a thread of its own, on
    a copy stream, starting before the plan is made. Each wedge goes in copies of `chunk` frames with at most `queued`
    copies waiting in the copy engine (it serves copies in submission order, across streams), so a small copy the
    integration issues meanwhile waits for little; at most `depth` wedges are held on the device."""

    def __init__(self, host, first, wedges, oks, device, depth=4, chunk=2, queued=4):
        self.host, self.first = host, first
        self.wedges, self.oks = wedges, oks
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(device=self.device)
        self.ready = [threading.Event() for _ in wedges]
        self.out = [None] * len(wedges)
        self.held = [False] * len(wedges)   # the wedge took a slot
        self.slots = threading.Semaphore(depth)
        self.chunk, self.queued = chunk, queued
        self.error = None
        self.stopping = False
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        try:
            torch.cuda.set_device(self.device)
            pend = collections.deque()
            with torch.cuda.stream(self.stream):
                for w, (fa, fb) in enumerate(self.wedges):
                    if not self.oks[w].any():
                        self.ready[w].set()
                        continue
                    self.slots.acquire()
                    if self.stopping:
                        break
                    self.held[w] = True
                    h = self.host[fa - self.first:fb - self.first + 1]
                    d = torch.empty(h.shape, dtype=h.dtype, device=self.device)
                    for c0 in range(0, h.shape[0], self.chunk):
                        while len(pend) >= self.queued:
                            ev0 = pend.popleft()
                            while not ev0.query():       # polling lets the integration's thread run meanwhile
                                time.sleep(2e-4)
                        d[c0:c0 + self.chunk].copy_(h[c0:c0 + self.chunk], non_blocking=True)
                        ev = torch.cuda.Event()
                        ev.record(self.stream)
                        pend.append(ev)
                    self.out[w] = (d, pend[-1])
                    self.ready[w].set()
        except BaseException as e:          # surfaced by get()
            self.error = e
            for r in self.ready:
                r.set()

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
    def __init__(self, data, first=1, overload=1 << 20, min_valid=0, device="cuda"):
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
        self._ring = _PinnedRing(torch.int32)

    def _host_slice(self, a, b):
        return self.data[a - self.first:b - self.first + 1]

    def feeder(self, wedges, oks):
        """A transfer thread for the run's wedges when the frames are a pinned host tensor (None otherwise)."""
        d = self.data
        if self.on_device or not torch.is_tensor(d) or not d.is_pinned():
            return None
        h = d if d.dtype == torch.int32 else d.view(torch.int32)
        return _Feeder(h, self.first, wedges, oks, self.device)

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
