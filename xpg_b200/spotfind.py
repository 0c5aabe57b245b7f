"""Strong-pixel classifier of spot finding on the device: XPG's `make_finder` (`xpg/spotfind.py:57-97`) with the same
arguments and results, computed by libxpgi.so (`xi_spot_strong`): the dispersion test (Kabsch 2010) and the extended
second pass, bit for bit with the reference on float32 frames (negative pixels are not valid)."""
from __future__ import annotations

import ctypes as C

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


def find_spots(img, gain=1.0, first_frame=0, finder=None, min_pix=1, max_pix=1000000, max_centroid_dist=3.0,
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
