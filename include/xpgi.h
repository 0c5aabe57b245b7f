/*
 * xpgi.h: C ABI of the B200 shoebox integration kernels (libxpgi.so).
 *
 * Every entry point takes plain device pointers and sizes, runs on the given CUDA stream and returns an int status:
 * XI_OK or one of the XI_E_* codes below (never a CUDA fault on bad sizes: shapes are checked on the host first).
 * Output memory is allocated by the caller; nothing here allocates device memory.
 *
 * The kernels replace the inner kernel surface of XPG's integration, `make_kernels(Dz, Dy, Dx, n_regions)` ->
 * (pass1, accumulate_profiles, pass2) (xpg/integrate_kernels.py:216-485), plus the host loops around them that XPG
 * runs in numpy: the frame gather (xpg/integrate.py:704-787), the binned-shoebox decode (xpg/shoebox.py:264-268)
 * and the profile finalisation (xpg/integrate.py:546-555). Unlike the reference, one call covers reflections of
 * any shoebox shape: rows carry their own depth, side and arena offsets.
 *
 * Layouts (all row-major, float32 unless stated):
 *   shoebox arena   row i occupies Dz[i] * bx[i] * bx[i] floats at sb_off[i]: frame-bin z, box row y, column x,
 *                   stored as value + 3 (0 = unrecorded, i.e. -3; -1 + 3 masked; -2 + 3 overloaded)
 *   per-pixel out   row i occupies bx[i]^2 values at pix_off[i] (img2, J, u1, u2, all_valid2)
 *   per-frame out   row i occupies Dz[i] values at frm_off[i] (fz)
 *   neighbours      (n, K) arrays, row-major
 *   profiles        (n_regions, 41, 41); accumulation grids num / den in float64
 */
#ifndef XPGI_H
#define XPGI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XI_OK 0
#define XI_E_ARG 1        /* a null pointer or a negative size */
#define XI_E_SHAPE 2      /* a shoebox shape outside the supported range */
#define XI_E_CUDA 3       /* a CUDA launch or runtime error (message: xi_last_error) */
#define XI_E_LIMIT 4      /* a size beyond a documented maximum */

#define XI_GRID 41        /* profile grid points per axis (PROFILE_GRID, xpg/integrate_kernels.py:18) */
#define XI_RC_K 21        /* rocking-curve mixture components (RC_C, xpg/integrate_kernels.py:121) */
#define XI_MAX_DZ 65      /* deepest shoebox (max(DZ_BUCKETS), xpg/integrate.py:44) */
#define XI_MAX_BX 97      /* widest shoebox side (max(XY_BUCKETS), xpg/integrate.py:47) */
#define XI_MAX_K 16       /* neighbour columns per reflection (8 + n_foreign, xpg/integrate.py:292, :303) */

/* Detector constants: XPG's _detector_consts (xpg/integrate_kernels.py:48-65). Device pointers. */
typedef struct {
    int n_panels;                   /* >= 1 */
    const float *P0, *Bx, *By;      /* (n_panels, 3) lab affine map per panel */
    const float *U1, *U2, *UN;      /* (n_panels, 3) panel axes and normal */
    const int16_t *segmap;          /* (seg_ny, seg_nx) panel of each pixel, -1 in gaps; NULL: single panel */
    int seg_nx, seg_ny;
    const float *gx, *gy;           /* (geo_ny, geo_nx) distortion tables (pixels); NULL: none */
    int geo_nx, geo_ny;
    const float *bkg;               /* (bkg_ny, bkg_nx) background template; NULL: flat */
    int bkg_nx, bkg_ny;
    float orgx, orgy, qx, qy, wl;   /* beam origin (pixels), pixel size (mm), wavelength (A) */
    float tsens, mu, inv_mu;        /* sensor thickness (mm), attenuation (1/mm) and 1/mu; used when parallax */
    int parallax;                   /* 1: invert thick-sensor parallax (2 iterations) */
} XiDetector;

/* Per-reflection inputs of a kernel call: XPG's `rc` and `nb` dicts (xpg/integrate.py:509-517). Device pointers. */
typedef struct {
    int n;                          /* rows */
    const float *S;                 /* (n, 3) diffracted wave vector */
    const float *phi;               /* (n) predicted spindle angle (radians) */
    const int32_t *ix0, *iy0;       /* (n) box origin in the row's (super-)pixel units */
    const int32_t *iz0;             /* (n) first frame index (0-based) */
    const float *fb;                /* (n) frames per phi bin */
    const int32_t *region;          /* (n) detector region of the reference profile */
    const float *has_p;             /* (n) 1: joint fit with the overlapping partner */
    const float *pS;                /* (n, 3) partner's S */
    const float *pphi;              /* (n) partner's phi */
    const int32_t *pxs;             /* (n) super-pixel side (1: none) */
    const int32_t *Dz, *bx;         /* (n) shoebox depth and side */
    const int64_t *sb_off;          /* (n) arena offset (floats) */
    const int64_t *pix_off;         /* (n) per-pixel output offset */
    const int64_t *frm_off;         /* (n) per-frame output offset */
    int K;                          /* neighbour columns */
    const float *nbx, *nby, *nbz, *nbsx, *nbsz;   /* (n, K) neighbour ellipsoids (pixels, frames) */
    const int32_t *order;           /* (n_order) rows processed by the call (NULL: rows 0..n-1) */
    int n_order;
    int max_bx, max_dz;             /* largest side / depth among the processed rows (sizes shared memory);
                                       rows beyond them are skipped and flagged (xi_status) */
    float sb_bias;                  /* voxel value = stored value - sb_bias (3 for the +3 arena, 0 for plain
                                       shoeboxes as XPG's kernels receive them) */
} XiRows;

/* Block constants of a kernel call (xpg/integrate.py:466-475). rcw: device (21). */
typedef struct {
    float frames_phi0;              /* spindle angle (radians) at frame coordinate 0 */
    float osc;                      /* radians per frame */
    float sd, sm;                   /* sigma_D, sigma_M (radians) */
    float gain;
    const float *rcw;               /* rocking-curve mixture weights */
    float s0[3], axis[3];           /* beam vector (1/A) and rotation axis */
} XiBlock;

/* Pass-1 outputs (xpg/integrate_kernels.py:362-365). Device pointers, caller-allocated. */
typedef struct {
    float *bg, *nbg, *isum, *vsum, *vsum0, *xo, *yo, *zo, *m_d, *m_m, *frac_rec, *nfg, *zeta, *seff;   /* (n) */
    int64_t *n_over, *n_fg_masked, *n_fg_nb;                                                         /* (n) */
    float *fz;                      /* per-frame */
    float *img2, *J, *u1, *u2;      /* per-pixel */
    uint8_t *all_valid2;            /* per-pixel */
} XiPass1Out;

/* Pass-1 inputs that pass 2 reuses (the `pix` argument, xpg/integrate.py:560-563) plus the background. */
typedef struct {
    const float *zeta, *seff, *J, *u1, *u2;   /* pass-1 outputs */
    const float *bg, *nbg;
} XiPass2In;

/* Pass-2 outputs (xpg/integrate_kernels.py:429, :482). Device pointers, caller-allocated, (n) each. */
typedef struct {
    float *iprf, *vprf, *vprf0, *corr, *p_valid, *p_total, *ipartner, *rho, *p_fg;
} XiPass2Out;

/* Rows of a gather call: the boxes of one phi block's reflections (xpg/integrate.py:372-398). Device pointers. */
typedef struct {
    int n;
    const int32_t *ix0, *iy0;       /* (super-)pixel units */
    const int32_t *iz0, *fb, *Dz, *bx, *pxs;
    const int64_t *sb_off;          /* arena offset (floats) */
    const int64_t *cnt_off;         /* offset of the row's Dz bin counters in `cnt` (binned rows), else -1 */
    const int32_t *order;           /* (n_order) rows processed by the call (NULL: rows 0..n-1) */
    int n_order;
} XiGatherRows;

/* Frames of a gather call. Frame w of the wedge is frame index first_fi + w (0-based). */
typedef struct {
    const void *data;               /* n_frames * ny * nx values: uint32 raw counts, or float32 prepared frames */
    int is_float;                   /* 0: raw uint32 (encoded here), 1: float32 already encoded (-1 / -2) */
    int n_frames, ny, nx;
    int first_fi;
    const uint8_t *frame_ok;        /* (n_frames) 0: frame excluded (never read); NULL: all read */
    uint32_t overload;              /* raw >= overload: -2 */
    uint32_t min_valid;             /* raw < min_valid: -1 (0: none) */
    const uint8_t *mask;            /* (ny, nx) 0 = masked (min(value, -1)); NULL: none */
} XiFrames;

/* Last error message of this thread (empty when none). */
const char *xi_last_error(void);
/* ABI version: increases when a signature above changes. */
int xi_version(void);
/* Synchronises the stream and reports (then clears) the kernels' status word: XI_E_SHAPE when a row was skipped
 * because its shape exceeded its call's max_bx / max_dz. */
int xi_status(void *stream);

/* Frame gather (xpg/integrate.py:704-787 with the preparation of :667-699 and the encoding of
 * xpg/io/images.py:72-102): every row's box window of every frame of the wedge inside its frame range is written
 * to its arena slot (value + 3), or, for binned rows (fb > 1), added to its bin in IEEE encoding (overloaded: NaN,
 * masked: +inf) with the bin's frame counter incremented. Frames must be passed in increasing order over calls. */
int xi_gather(const XiFrames *frames, const XiGatherRows *rows, float *arena, int32_t *cnt, void *stream);

/* Binned-bin decode (xpg/shoebox.py:264-268, xpg/integrate.py:483-488): NaN -> -2, inf -> -1, stored + 3; bins
 * with fewer than fb frames recorded become unrecorded (0). Applies to rows with cnt_off >= 0. */
int xi_decode_bins(const XiGatherRows *rows, float *arena, const int32_t *cnt, void *stream);

/* Pass 1 (xpg/integrate_kernels.py:287-365): pixel geometry, masks, robust background, summation, centroids,
 * moments and the projected 2D spot of every row. */
int xi_pass1(const XiDetector *det, const XiRows *rows, const XiBlock *blk, const float *arena, XiPass1Out *out,
             void *stream);

/* Profile accumulation (xpg/integrate_kernels.py:367-380): selected rows scatter their normalised projected spot
 * bilinearly into num / den (float64, accumulated onto what they hold). strong_test = 1 applies the strong-row test
 * of xpg/integrate.py:531-533 (reads isum, vsum, n_over, frac_rec, n_fg_nb, n_fg_masked); sel: (n) optional extra
 * row selection (NULL: all rows). Reads img2, all_valid2, J, u1, u2, isum, seff. */
int xi_accumulate(const XiRows *rows, const XiPass1Out *p1, const uint8_t *sel, int strong_test, int n_regions,
                  double *num, double *den, void *stream);

/* Profile finalisation (xpg/integrate.py:546-555): prof = (den * max(num / den, 0) + 3 * gauss) / (den + 3),
 * normalised to unit integral, per region. */
int xi_finalize_profiles(const double *num, const double *den, int n_regions, float *prof, void *stream);

/* Pass 2 (xpg/integrate_kernels.py:382-483): profile fit with fixed background, joint fit with the overlapping
 * partner, variances, correlation and recorded fractions. prof: (n_regions, 41, 41). */
int xi_pass2(const XiDetector *det, const XiRows *rows, const XiBlock *blk, const float *arena, const float *prof,
             const XiPass2In *in, XiPass2Out *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
