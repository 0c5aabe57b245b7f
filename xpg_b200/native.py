"""ctypes binding of libxpgi.so (include/xpgi.h): structs and thin callers that take torch CUDA tensors.

The library is the product's only compute path: a missing library or a missing GPU raises at once; there is no
fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libxpgi.so"

XI_OK, XI_E_ARG, XI_E_SHAPE, XI_E_CUDA, XI_E_LIMIT = 0, 1, 2, 3, 4
XI_GRID, XI_RC_K, XI_MAX_DZ, XI_MAX_BX, XI_MAX_K = 41, 21, 65, 97, 16

_fp = C.c_void_p      # every device pointer travels as void*


class XiDetector(C.Structure):
    _fields_ = [("n_panels", C.c_int), ("P0", _fp), ("Bx", _fp), ("By", _fp), ("U1", _fp), ("U2", _fp),
                ("UN", _fp), ("segmap", _fp), ("seg_nx", C.c_int), ("seg_ny", C.c_int), ("gx", _fp), ("gy", _fp),
                ("geo_nx", C.c_int), ("geo_ny", C.c_int), ("bkg", _fp), ("bkg_nx", C.c_int), ("bkg_ny", C.c_int),
                ("orgx", C.c_float), ("orgy", C.c_float), ("qx", C.c_float), ("qy", C.c_float), ("wl", C.c_float),
                ("tsens", C.c_float), ("mu", C.c_float), ("inv_mu", C.c_float), ("parallax", C.c_int)]


class XiRows(C.Structure):
    _fields_ = [("n", C.c_int), ("S", _fp), ("phi", _fp), ("ix0", _fp), ("iy0", _fp), ("iz0", _fp), ("fb", _fp),
                ("region", _fp), ("has_p", _fp), ("pS", _fp), ("pphi", _fp), ("pxs", _fp), ("Dz", _fp),
                ("bx", _fp), ("sb_off", _fp), ("pix_off", _fp), ("frm_off", _fp), ("K", C.c_int), ("nbx", _fp),
                ("nby", _fp), ("nbz", _fp), ("nbsx", _fp), ("nbsz", _fp), ("order", _fp), ("n_order", C.c_int),
                ("max_bx", C.c_int), ("max_dz", C.c_int), ("sb_bias", C.c_float)]


class XiBlock(C.Structure):
    _fields_ = [("frames_phi0", C.c_float), ("osc", C.c_float), ("sd", C.c_float), ("sm", C.c_float),
                ("gain", C.c_float), ("rcw", _fp), ("s0", C.c_float * 3), ("axis", C.c_float * 3)]


class XiPass1Out(C.Structure):
    _fields_ = [(k, _fp) for k in ("bg", "nbg", "isum", "vsum", "vsum0", "xo", "yo", "zo", "m_d", "m_m",
                                   "frac_rec", "nfg", "zeta", "seff", "n_over", "n_fg_masked", "n_fg_nb", "fz",
                                   "img2", "J", "u1", "u2", "all_valid2")]


class XiPass2In(C.Structure):
    _fields_ = [(k, _fp) for k in ("zeta", "seff", "J", "u1", "u2", "bg", "nbg")]


class XiPass2Out(C.Structure):
    _fields_ = [(k, _fp) for k in ("iprf", "vprf", "vprf0", "corr", "p_valid", "p_total", "ipartner", "rho",
                                   "p_fg")]


class XiGatherRows(C.Structure):
    _fields_ = [("n", C.c_int), ("ix0", _fp), ("iy0", _fp), ("iz0", _fp), ("fb", _fp), ("Dz", _fp), ("bx", _fp),
                ("pxs", _fp), ("sb_off", _fp), ("cnt_off", _fp), ("order", _fp), ("n_order", C.c_int)]


class XiFrames(C.Structure):
    _fields_ = [("data", _fp), ("is_float", C.c_int), ("n_frames", C.c_int), ("ny", C.c_int), ("nx", C.c_int),
                ("first_fi", C.c_int), ("frame_ok", _fp), ("overload", C.c_uint32), ("min_valid", C.c_uint32),
                ("mask", _fp)]


class XiSynthSpots(C.Structure):
    _fields_ = [("n", C.c_int), ("x", _fp), ("y", _fp), ("z", _fp), ("counts", _fp), ("sig_t", _fp),
                ("sig_r", _fp), ("sig_z", _fp), ("orgx", C.c_double), ("orgy", C.c_double)]


class XiSynthBackground(C.Structure):
    _fields_ = [("level", C.c_double), ("ramp", C.c_double), ("orgx", C.c_double), ("orgy", C.c_double),
                ("rmax", C.c_double)]


EXPORTS = ("xi_last_error", "xi_version", "xi_status", "xi_gather", "xi_decode_bins", "xi_pass1", "xi_accumulate",
           "xi_finalize_profiles", "xi_pass2")

_LIB = None


def load(path=None):
    """The loaded library (built in-tree by xpg_b200.csrc.build)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m xpg_b200.csrc.build`")
    lib = C.CDLL(str(p))
    lib.xi_last_error.restype = C.c_char_p
    lib.xi_version.restype = C.c_int
    for name in EXPORTS[2:]:
        getattr(lib, name).restype = C.c_int
    lib.xi_status.argtypes = [C.c_void_p]
    lib.xi_gather.argtypes = [C.POINTER(XiFrames), C.POINTER(XiGatherRows), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_decode_bins.argtypes = [C.POINTER(XiGatherRows), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_pass1.argtypes = [C.POINTER(XiDetector), C.POINTER(XiRows), C.POINTER(XiBlock), C.c_void_p,
                             C.POINTER(XiPass1Out), C.c_void_p]
    lib.xi_accumulate.argtypes = [C.POINTER(XiRows), C.POINTER(XiPass1Out), C.c_void_p, C.c_int, C.c_int,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_finalize_profiles.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.xi_pass2.argtypes = [C.POINTER(XiDetector), C.POINTER(XiRows), C.POINTER(XiBlock), C.c_void_p, C.c_void_p,
                             C.POINTER(XiPass2In), C.POINTER(XiPass2Out), C.c_void_p]
    lib.xi_synth_frames.restype = C.c_int
    lib.xi_synth_frames.argtypes = [C.POINTER(XiSynthSpots), C.POINTER(XiSynthBackground), C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p]
    lib.xi_synth_last_error.restype = C.c_char_p
    if path is None:
        _LIB = lib
    return lib


def check(rc, what):
    if rc != XI_OK:
        msg = load().xi_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed (status {rc}): {msg}")


def ptr(t):
    """Device address of a tensor (None -> NULL). The tensor must stay alive across the call."""
    if t is None:
        return None
    if not t.is_cuda:
        raise RuntimeError("xpg_b200 kernels take CUDA tensors only (no CPU path)")
    return C.c_void_p(t.data_ptr())


def stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("xpg_b200 needs a CUDA device: the integration kernels have no CPU path")
    load()
