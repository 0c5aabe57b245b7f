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
                                   "img2", "J", "u1", "u2", "all_valid2", "isum_raw")]


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
    _fields_ = [("n", C.c_int), ("index", _fp), ("x", _fp), ("y", _fp), ("z", _fp), ("counts", _fp), ("sig_t", _fp),
                ("sig_r", _fp), ("sig_z", _fp), ("orgx", C.c_double), ("orgy", C.c_double)]


class XiSynthBackground(C.Structure):
    _fields_ = [("level", C.c_double), ("ramp", C.c_double), ("orgx", C.c_double), ("orgy", C.c_double),
                ("rmax", C.c_double)]


class XiFmBoxes(C.Structure):
    _fields_ = [("n", C.c_int), ("n_terms", C.c_int), ("Dz", C.c_int), ("b", C.c_int), ("R", C.c_void_p),
                ("P", C.c_void_p), ("iz0", C.c_void_p), ("iy0", C.c_void_p), ("ix0", C.c_void_p)]


class XiFmWindow(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("f0", "nf", "y0", "ny", "x0", "nx")]


XI_FM_NS_I16, XI_FM_NS_I32, XI_FM_NS_F32 = 0, 1, 2
XI_PANEL_F64 = 28
XI_PANELS_INLINE = 4
XI_KNN_MAX = 16
XI_KNN_NOALLOC_MAX_POINTS, XI_KNN_NOALLOC_MAX_CELLS = 1 << 19, 1 << 18
_d3 = C.c_double * 3


class XiPlanDetector(C.Structure):
    _fields_ = [("n_panels", C.c_int), ("panels", _fp), ("segmented", C.c_int), ("segmap", _fp),
                ("seg_nx", C.c_int), ("seg_ny", C.c_int), ("geo_x", _fp), ("geo_y", _fp), ("geo_nx", C.c_int),
                ("geo_ny", C.c_int), ("parallax", C.c_int), ("tsens", C.c_double), ("mu", C.c_double),
                ("orgx", C.c_double), ("orgy", C.c_double), ("qx", C.c_double), ("qy", C.c_double),
                ("distance", C.c_double), ("ed1", _d3), ("ed2", _d3), ("ed3", _d3), ("beam", _d3), ("pol_n", _d3),
                ("pol_main", _d3), ("pol_f", C.c_double), ("nx", C.c_double), ("ny", C.c_double),
                ("panel_inline", C.c_double * (4 * 28))]


class XiPredict(C.Structure):
    _fields_ = [("astar", C.c_double * 9), ("hmax", C.c_int * 3), ("q2_max", C.c_double), ("q2_min", C.c_double),
                ("centring", C.c_int), ("hkl", _fp), ("n_hkl", C.c_int64), ("axis", _d3),
                ("rot_K", C.c_double * 9), ("rot_kk", C.c_double * 9), ("s0", _d3), ("phi_lo", C.c_double),
                ("phi_hi", C.c_double), ("phi0", C.c_double), ("osc", C.c_double), ("z_shift", C.c_double),
                ("deg", C.c_double), ("rad", C.c_double), ("acc_s0", _d3), ("acc_axis", _d3),
                ("min_zeta", C.c_double), ("x_hi", C.c_double), ("y_hi", C.c_double), ("z_lo", C.c_double),
                ("z_hi", C.c_double), ("block", C.c_int), ("lattice", C.c_int)]


class XiPredictOut(C.Structure):
    _fields_ = [(k, _fp) for k in ("hkl", "phi", "S", "x", "y", "z", "zeta", "polarization", "zeta_k", "block",
                                   "lattice")]


class XiBoxRules(C.Structure):
    _fields_ = [("n", C.c_int64), ("x", _fp), ("y", _fp), ("z", _fp), ("zeta_k", _fp), ("sigma_m", C.c_double),
                ("abs_osc", C.c_double), ("osc2_12", C.c_double), ("rsd_box", C.c_double), ("rsd", C.c_double),
                ("qmin", C.c_double), ("box", C.c_int), ("box_fixed", C.c_int), ("n_xyb", C.c_int),
                ("xyb", C.c_int * 16), ("f_first", C.c_int), ("f_last", C.c_int), ("n_regions_xy", C.c_int)]


class XiBoxOut(C.Structure):
    _fields_ = [(k, _fp) for k in ("iz0", "dz", "fb", "Dz", "bx", "pxs", "ix0", "iy0", "region", "zstart", "zend",
                                   "flags", "coverage", "sx_px", "sz_f")]


class XiKnn(C.Structure):
    _fields_ = [("n", C.c_int64), ("x", _fp), ("y", _fp), ("z", _fp), ("sx", C.c_double), ("sz", C.c_double),
                ("lo", _d3), ("hi", _d3), ("radius", C.c_double), ("k", C.c_int)]


class XiRocking(C.Structure):
    _fields_ = [("n", C.c_int64), ("fz", _fp), ("iz0", _fp), ("phi", _fp), ("zeta", _fp), ("phi0", C.c_double),
                ("osc", C.c_double), ("z_shift", C.c_double)]


class XiSpotParams(C.Structure):
    _fields_ = [("nbx", C.c_int), ("nby", C.c_int), ("signal_pixel", C.c_float), ("background_pixel", C.c_float),
                ("min_local", C.c_int), ("extended", C.c_int)]


XI_SPOT_MAX_HALF = 8


class XiPackedFrame(C.Structure):
    _fields_ = [("plane", _fp), ("exc", _fp), ("n_exc", C.c_int64), ("raw", C.c_int)]


class XiGatherStep(C.Structure):
    _fields_ = [("frames", XiFrames), ("order", _fp), ("n_order", C.c_int)]


class XiRowSet(C.Structure):
    _fields_ = [("det", XiDetector), ("rows", XiRows), ("blk", XiBlock), ("arena", _fp), ("p1", XiPass1Out),
                ("prof", _fp), ("p2", XiPass2Out)]


class XiHklRows(C.Structure):
    _fields_ = [("n", C.c_int64), ("hkl", C.c_void_p), ("I", C.c_void_p), ("sig", C.c_void_p), ("x", C.c_void_p),
                ("y", C.c_void_p), ("zc", C.c_void_p), ("rlp", C.c_void_p), ("peak", C.c_void_p),
                ("corr", C.c_void_p), ("xo", C.c_void_p), ("yo", C.c_void_p), ("zo", C.c_void_p),
                ("alf1", C.c_void_p), ("bet1", C.c_void_p), ("alf0", C.c_double), ("bet0", C.c_double)]


XI_TUNE_PASS1_STAGE_BYTES, XI_TUNE_PASS2_STAGE_BYTES, XI_TUNE_PASS2_LIST_CAP, XI_TUNE_WIDE_THREADS = 1, 2, 3, 4
XI_TUNE_PASS2_LIST_CAP_LARGE, XI_PASS2_LARGE_VOXELS = 5, 49152
XI_PACK_ESCAPE, XI_PACK_FLAGGED = 254, 255

EXPORTS = ("xi_last_error", "xi_version", "xi_status", "xi_status_copy", "xi_tune", "xi_gather", "xi_decode_bins",
           "xi_pass1", "xi_accumulate", "xi_finalize_profiles", "xi_pass2", "xi_predict_count", "xi_predict_write",
           "xi_plan_boxes", "xi_knn", "xi_knn_noalloc", "xi_rocking_costs", "xi_rocking_gram",
           "xi_predict_workspace", "xi_knn_workspace", "xi_rocking_gram_workspace", "xi_pack_u8", "xi_unpack_u8",
           "xi_upload", "xi_bslz4_lz4_stage", "xi_bitunshuffle", "xi_format_integrate_hkl", "xi_spot_strong",
           "xi_spot_workspace", "xi_pass1_batched", "xi_pass2_batched", "xi_gather_step", "xi_unpack_u8_frames",
           "xi_zero_rows", "xi_fm_scatter", "xi_fm_gather")

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
    lib.xi_predict_workspace.restype = C.c_size_t
    lib.xi_knn_workspace.restype = C.c_size_t
    lib.xi_predict_workspace.argtypes = [C.POINTER(XiPredict)]
    lib.xi_predict_count.argtypes = [C.POINTER(XiPredict), C.POINTER(XiPlanDetector), C.c_void_p, C.c_size_t,
                                     C.POINTER(C.c_int64), C.c_void_p]
    lib.xi_predict_write.argtypes = [C.POINTER(XiPredict), C.POINTER(XiPlanDetector), C.c_void_p, C.c_size_t,
                                     C.POINTER(XiPredictOut), C.c_int64, C.c_void_p]
    lib.xi_plan_boxes.argtypes = [C.POINTER(XiBoxRules), C.POINTER(XiPlanDetector), C.POINTER(XiBoxOut), C.c_void_p]
    lib.xi_knn_workspace.argtypes = [C.POINTER(XiKnn)]
    lib.xi_knn.argtypes = [C.POINTER(XiKnn), C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_knn_noalloc.argtypes = [C.POINTER(XiKnn), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_rocking_costs.argtypes = [C.POINTER(XiRocking), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.xi_rocking_gram_workspace.restype = C.c_size_t
    lib.xi_rocking_gram_workspace.argtypes = [C.POINTER(XiRocking)]
    lib.xi_rocking_gram.argtypes = [C.POINTER(XiRocking), C.c_double, C.c_void_p, C.c_size_t, C.c_void_p,
                                    C.c_void_p, C.c_void_p]
    lib.xi_pack_u8.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                               C.POINTER(C.c_int64)]
    lib.xi_unpack_u8.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    lib.xi_upload.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    lib.xi_bslz4_lz4_stage.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int64, C.c_int,
                                       C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.xi_bitunshuffle.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int64, C.c_void_p, C.c_void_p]
    lib.xi_spot_workspace.restype = C.c_size_t
    lib.xi_spot_workspace.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.xi_spot_strong.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(XiSpotParams),
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
    lib.xi_format_integrate_hkl.argtypes = [C.POINTER(XiHklRows), C.c_void_p, C.c_int64, C.c_int,
                                            C.POINTER(C.c_int64)]
    lib.xi_status.argtypes = [C.c_void_p]
    lib.xi_status_copy.argtypes = [C.c_void_p, C.c_void_p]
    lib.xi_tune.argtypes = [C.c_int, C.c_longlong]
    lib.xi_gather.argtypes = [C.POINTER(XiFrames), C.POINTER(XiGatherRows), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_decode_bins.argtypes = [C.POINTER(XiGatherRows), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_zero_rows.argtypes = [C.POINTER(XiGatherRows), C.c_void_p, C.c_void_p]
    lib.xi_pass1.argtypes = [C.POINTER(XiDetector), C.POINTER(XiRows), C.POINTER(XiBlock), C.c_void_p,
                             C.POINTER(XiPass1Out), C.c_void_p]
    lib.xi_accumulate.argtypes = [C.POINTER(XiRows), C.POINTER(XiPass1Out), C.c_void_p, C.c_int, C.c_int,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
    lib.xi_finalize_profiles.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.xi_pass2.argtypes = [C.POINTER(XiDetector), C.POINTER(XiRows), C.POINTER(XiBlock), C.c_void_p, C.c_void_p,
                             C.POINTER(XiPass2In), C.POINTER(XiPass2Out), C.c_void_p]
    lib.xi_unpack_u8_frames.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
    lib.xi_gather_step.argtypes = [C.c_void_p, C.POINTER(XiGatherRows), C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_void_p]
    for name in ("xi_pass1_batched", "xi_pass2_batched"):
        getattr(lib, name).argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.c_void_p]
    lib.xi_synth_frames.restype = C.c_int
    lib.xi_synth_frames.argtypes = [C.POINTER(XiSynthSpots), C.POINTER(XiSynthBackground), C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p]
    lib.xi_synth_last_error.restype = C.c_char_p
    lib.xi_fm_last_error.restype = C.c_char_p
    lib.xi_fm_scatter.argtypes = [C.POINTER(XiFmBoxes), C.POINTER(XiFmWindow), C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p]
    lib.xi_fm_gather.argtypes = [C.POINTER(XiFmBoxes), C.POINTER(XiFmWindow), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    if path is None:
        _LIB = lib
        _apply_tuned(lib)
    return lib


def _apply_tuned(lib):
    """The launch shape measured best on this device by xpg_b200.tune (tuned.json), when there is one."""
    try:
        from .tune import load_shape
        shape = load_shape()
    except Exception:
        shape = None
    if not shape:
        return
    keys = {"wide_threads": XI_TUNE_WIDE_THREADS, "pass1_stage_bytes": XI_TUNE_PASS1_STAGE_BYTES,
            "pass2_stage_bytes": XI_TUNE_PASS2_STAGE_BYTES, "pass2_list_cap": XI_TUNE_PASS2_LIST_CAP,
            "pass2_list_cap_large": XI_TUNE_PASS2_LIST_CAP_LARGE}
    for k, v in shape.items():
        if k in keys:
            lib.xi_tune(keys[k], int(v))


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


def tune(pass1_stage_bytes=None, pass2_stage_bytes=None, pass2_list_cap=None, wide_threads=None,
         pass2_list_cap_large=None):
    """Launch tuning of the pass kernels (results are independent of it)."""
    lib = load()
    if pass2_list_cap_large is not None:
        check(lib.xi_tune(XI_TUNE_PASS2_LIST_CAP_LARGE, int(pass2_list_cap_large)), "xi_tune")
    if wide_threads is not None:
        check(lib.xi_tune(XI_TUNE_WIDE_THREADS, int(wide_threads)), "xi_tune")
    if pass1_stage_bytes is not None:
        check(lib.xi_tune(XI_TUNE_PASS1_STAGE_BYTES, int(pass1_stage_bytes)), "xi_tune")
    if pass2_stage_bytes is not None:
        check(lib.xi_tune(XI_TUNE_PASS2_STAGE_BYTES, int(pass2_stage_bytes)), "xi_tune")
    if pass2_list_cap is not None:
        check(lib.xi_tune(XI_TUNE_PASS2_LIST_CAP, int(pass2_list_cap)), "xi_tune")
