"""Strong-pixel classifier of spot finding on the device: XPG's `make_finder` (`xpg/spotfind.py:57-97`) with the same
arguments and results, computed by libxpgi.so (`xi_spot_strong`): the dispersion test (Kabsch 2010) and the extended
second pass, bit for bit with the reference on float32 frames (negative pixels are not valid)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import native as N


def make_finder(nbx=3, nby=3, signal_pixel=3.0, background_pixel=2.0, min_local=2, extended=True):
    """find(img, gain) -> (strong, mean): img a (B, ny, nx) or (ny, nx) float32 CUDA tensor; strong bool and mean
    float32 of the same shape."""
    p = N.XiSpotParams()
    p.nbx, p.nby = int(nbx), int(nby)
    p.signal_pixel, p.background_pixel = float(signal_pixel), float(background_pixel)
    p.min_local, p.extended = int(min_local), 1 if extended else 0

    @torch.no_grad()
    def find(img, gain):
        if not img.is_cuda:
            raise RuntimeError("xpg_b200 spot finding takes CUDA tensors only (no CPU path)")
        x = img.to(torch.float32).contiguous()
        shape = x.shape
        if x.dim() == 2:
            x = x[None]
        B, ny, nx = (int(v) for v in x.shape)
        strong = torch.empty((B, ny, nx), dtype=torch.uint8, device=x.device)
        mean = torch.empty((B, ny, nx), dtype=torch.float32, device=x.device)
        lib = N.load()
        nws = int(lib.xi_spot_workspace(B, ny, nx)) if extended else 0
        ws = torch.empty(max(nws, 1), dtype=torch.uint8, device=x.device)
        N.check(lib.xi_spot_strong(N.ptr(x), B, ny, nx, float(gain), C.byref(p), N.ptr(strong), N.ptr(mean),
                                   N.ptr(ws), nws, N.stream_handle()), "xi_spot_strong")
        return strong.bool().reshape(shape), mean.reshape(shape)

    return find


@dataclass
class SpotList:
    """Spots as XPG's `SpotList` holds them (`xpg/spotcluster.py:20-46`): pixel coordinates, continuous frame
    coordinate (frame f covers [f - 1, f)), background-subtracted intensity, pixel count, frame range."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    intensity: np.ndarray
    npix: np.ndarray
    zmin: np.ndarray
    zmax: np.ndarray
    hkl: np.ndarray | None = None

    def __len__(self):
        return self.x.size

    def subset(self, sel):
        return SpotList(**{k: (v[sel] if v is not None else None) for k, v in self.__dict__.items()})

    def write_legacy_spots(self, path):
        """SPOT.XDS records: x, y, z (10.2f), intensity (10.0f and a point), the indices when assigned."""
        with open(path, "w") as f:
            for i in range(len(self)):
                line = f"{self.x[i]:10.2f}{self.y[i]:10.2f}{self.z[i]:10.2f}{self.intensity[i]:10.0f}."
                if self.hkl is not None:
                    line += f"{self.hkl[i, 0]:8d}{self.hkl[i, 1]:8d}{self.hkl[i, 2]:8d}"
                f.write(line + "\n")


def find_spots(images, frames, gain=1.0, mask=None, strong_pixel=3.0, background_pixel=2.0, min_pixels=6,
               max_pixels=5000, nbx=3, nby=3, batch=8, extended=True, verbose=True, max_centroid_dist=3.0,
               cluster_radius=2, log=print, finder=None, device="cuda"):
    """XPG's `find_spots` (`xpg/spotfind.py:122-300`) with its arguments and result: frames (1-based numbers) of an
    image set (`get(frame)` -> float32 frame, -1 masked / -2 overloaded) in batches of `batch` on the device, masked
    (`mask`: True = trusted), classified (`make_finder`, or `finder`), the strong pixels read back and clustered on the
    host all at once, the spots in the order XPG's streaming clustering emits them for these batches."""
    from .spotcluster import cluster_spots, streaming_order
    import time
    frames = [int(f) for f in frames]
    if any(b <= a for a, b in zip(frames, frames[1:])):
        # XPG's streaming accumulator closes its clusters at every break in the frame list; clustering all strong
        # pixels at once links frames by their numbers, which matches it only for increasing frame lists
        raise ValueError("find_spots: frame numbers must be strictly increasing")
    t0 = time.time()
    finder = finder or make_finder(nbx, nby, strong_pixel, background_pixel, extended=extended)
    nx, ny = int(images.nx), int(images.ny)
    mask_t = torch.as_tensor(np.asarray(mask), device=device) if mask is not None else None
    a = torch.full((batch, ny, nx), -1.0, dtype=torch.float32, device=device)
    parts, batches = [], []
    for i in range(0, len(frames), batch):
        fr = frames[i:i + batch]
        for j, f in enumerate(fr):
            a[j].copy_(torch.from_numpy(np.ascontiguousarray(images.get(f), np.float32)))
        if len(fr) < batch:
            a[len(fr):] = -1.0
        x = torch.where(mask_t[None], a, -1.0) if mask_t is not None else a
        strong, mean = finder(x, float(gain))
        kk, yy, xx = torch.nonzero(strong, as_tuple=True)
        val, bg = x[kk, yy, xx], mean[kk, yy, xx]
        kk, yy, xx, val, bg = (t.cpu().numpy() for t in (kk, yy, xx, val, bg))
        parts.append((np.asarray(fr, np.int64)[kk] - 1, yy, xx, val, bg))
        batches.append(fr)
    z, y, x_, v, b = (np.concatenate([p[k] for p in parts]) if parts else np.zeros(0) for k in range(5))
    sp = cluster_spots(z, y, x_, v, b, nx, ny, min_pixels, max_pixels, max_centroid_dist, cluster_radius,
                       with_parents=True)
    order = streaming_order(sp, batches)
    spots = SpotList(**{k: sp[k][order] for k in ("x", "y", "z", "intensity", "npix", "zmin", "zmax")})
    if verbose:
        log(f"  SPOTS: {len(spots)} spots from {z.size} strong pixels in {time.time() - t0:.1f}s")
    return spots


def spots_of_stack(img, gain=1.0, first_frame=0, finder=None, min_pix=1, max_pix=1000000, max_centroid_dist=3.0,
                   cluster_radius=2, **finder_args):
    """Spots of a stack of frames img (n, ny, nx) float32 (negative: not valid), frame index first_frame + k for
    img[k]: the strong pixels of the device classifier (`make_finder(**finder_args)` unless `finder` is given),
    read back, then clustered on the host (`spotcluster.cluster_spots`, XPG's clustering all at once). Returns the
    spot arrays x, y (pixels), z (frame coordinate), intensity, npix, zmin, zmax as XPG's `SpotList` holds them."""
    from .spotcluster import cluster_spots
    finder = finder or make_finder(**finder_args)
    strong, mean = finder(img, float(gain))
    k, y, x = torch.nonzero(strong, as_tuple=True)
    v, b = img[k, y, x], mean[k, y, x]
    k, y, x, v, b = (t.cpu().numpy() for t in (k, y, x, v, b))
    return cluster_spots(k + int(first_frame), y, x, v, b, int(img.shape[2]), int(img.shape[1]), min_pix, max_pix,
                         max_centroid_dist, cluster_radius)
