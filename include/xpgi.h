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
    int64_t *isum_raw;              /* (n) raw summed counts: the recorded counts of the summation voxels (foreground,
                                       valid, not a neighbour's), an exact integer sum; no counterpart output in XPG,
                                       whose float32 `vsum` holds gain times the same sum (xpg/integrate_kernels.py:
                                       318-329) */
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
/* ABI version: increases when a signature or struct above changes (3: XiPass1Out.isum_raw, XiRowSet). */
int xi_version(void);
/* Synchronises the stream and reports (then clears) the kernels' status word: XI_E_SHAPE when a row was skipped
 * because its shape exceeded its call's max_bx / max_dz. */
int xi_status(void *stream);
/* Queues a copy of the kernels' status word into host_dst (pinned host memory) on the stream, without waiting: the
 * caller reads it once the stream has passed that point; nonzero: a row was skipped (xi_status then reports and
 * clears it). */
int xi_status_copy(int *host_dst, void *stream);

/* Launch tuning (process-wide; no counterpart in XPG, whose torch kernels have no launch shape): the largest
 * shoebox (bytes) pass 1 / pass 2 stage in shared memory, pass 2's fit-list capacity (voxels) for launches whose
 * largest box is up to XI_PASS2_LARGE_VOXELS voxels and XI_PASS2_LARGE_DEPTH bins deep and for larger ones, and the
 * CTA width of large boxes. Results do not depend on these. */
#define XI_TUNE_PASS1_STAGE_BYTES 1
#define XI_TUNE_PASS2_STAGE_BYTES 2
#define XI_TUNE_PASS2_LIST_CAP 3
#define XI_TUNE_WIDE_THREADS 4      /* threads per CTA of the pass kernels for boxes over 200 pixels: 128 or 256 */
#define XI_TUNE_PASS2_LIST_CAP_LARGE 5
#define XI_PASS2_LARGE_VOXELS 49152
#define XI_PASS2_LARGE_DEPTH 33
int xi_tune(int key, long long value);

/* Frame gather (xpg/integrate.py:704-787 with the preparation of :667-699 and the encoding of
 * xpg/io/images.py:72-102): every row's box window of every frame of the wedge inside its frame range is written
 * to its arena slot (value + 3), or, for binned rows (fb > 1), added to its bin in IEEE encoding (overloaded: NaN,
 * masked: +inf) with the bin's frame counter incremented. Frames must be passed in increasing order over calls. */
int xi_gather(const XiFrames *frames, const XiGatherRows *rows, float *arena, int32_t *cnt, void *stream);

/* The gather of one wedge described in device memory (read when the kernel runs), for a launch captured once in a
 * CUDA graph and replayed for every wedge of a block: write the wedge's descriptor, then replay. The rows' boxes
 * (rows, arena, cnt) are fixed for the block; CTAs (grid) stride over the descriptor's rows. Same results as
 * xi_gather with those frames and rows. No counterpart in XPG (its gather is a host loop). */
typedef struct {
    XiFrames frames;                /* the wedge (data, first_fi, n_frames, ...); n_frames 0: nothing to gather */
    const int32_t *order;           /* (n_order) rows of the block gathered from this wedge, device */
    int n_order;
} XiGatherStep;

int xi_gather_step(const XiGatherStep *step, const XiGatherRows *rows, float *arena, int32_t *cnt, int grid,
                   void *stream);

/* Binned-bin decode (xpg/shoebox.py:264-268, xpg/integrate.py:483-488): NaN -> -2, inf -> -1, stored + 3; bins
 * with fewer than fb frames recorded become unrecorded (0). Applies to rows with cnt_off >= 0 (of rows->order when
 * given), once each, after their last frame has been gathered. */
int xi_decode_bins(const XiGatherRows *rows, float *arena, const int32_t *cnt, void *stream);

/* Zeroes the arena slots (Dz * bx^2 floats, rounded up to 4; 0 = unrecorded) of the rows (of rows->order when
 * given): the rows a block's gathers do not write in full (binned rows, which accumulate; rows whose frames reach
 * beyond the integrated range). XPG allocates its buffers zeroed (xpg/integrate.py:372-398); here the other rows'
 * slots are written whole by the gathers, so only these need clearing. `arena` on 16 bytes. */
int xi_zero_rows(const XiGatherRows *rows, float *arena, void *stream);

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

/* ---- Batched passes: rows of many phi blocks and sweeps in one persistent launch ------------------------------
 * XPG runs its kernels per shoebox shape and chunk of at most 8192 rows of one block (`process_block`'s chunk loop,
 * xpg/integrate.py:463-520, `_chunk_size` :145-148, the per-shape kernel cache :347-351). Here one launch takes the
 * rows of any phi blocks of any sweeps whose boxes fit a size bin: resident CTAs (as many as the SMs hold) take
 * (set, row) items from a device queue until it is empty, with the same per-row arithmetic and results as
 * xi_pass1 / xi_pass2. A set is one block's rows with that block's detector, constants, arena and buffers. */
typedef struct {
    XiDetector det;
    XiRows rows;                    /* order, n_order, max_bx, max_dz are not used: the items name the rows */
    XiBlock blk;                    /* pass 2: the widths adapted for the block's pass 2 */
    const float *arena;
    XiPass1Out p1;                  /* pass 1 writes these; pass 2 reads zeta, seff, J, u1, u2, bg and nbg */
    const float *prof;              /* pass 2: the block's profiles (n_regions, 41, 41) */
    XiPass2Out p2;                  /* pass 2 writes these */
} XiRowSet;

/* sets: device array; items: (n_items) int64 set << 32 | row, device, in the order CTAs take them (largest boxes
 * first balances the launch); every item's box must fit max_bx / max_dz and its set's K <= max_k (others are skipped
 * and flagged for xi_status); queue: one device int, reset by the call. */
int xi_pass1_batched(const XiRowSet *sets, const int64_t *items, int n_items, int max_bx, int max_dz, int max_k,
                     int *queue, void *stream);
int xi_pass2_batched(const XiRowSet *sets, const int64_t *items, int n_items, int max_bx, int max_dz, int max_k,
                     int *queue, void *stream);

/* ---- Planning: predictions, shoebox boxes and neighbour lists (float64) -------------------------------------
 * XPG plans an integration run in numpy on the host (xpg/integrate.py:222-316 with the predictions of
 * xpg/geometry.py:468-545 and the neighbour search of xpg/integrate.py:164-172); these entry points do the same on
 * the device. Row order is the reference's: block by block, then solution (phi_a, phi_b), then turn (0, +360 deg),
 * then Miller-index order (h slowest, l fastest on the generated grid; list order for an explicit list). Device
 * workspace is the caller's (sizes from the *_workspace functions). */

#define XI_PANEL_F64 28           /* doubles per panel record of XiPlanDetector.panels */

/* Detector of the planner (xpg/geometry.py:246-410; the panel maps of xpg/detector.py:79-90). Panel record k:
 * P0[3] Bx[3] By[3] n[3] u1[3] u2[3] un[3] P0.n Bx.Bx By.By x1 x2 y1 y2 with n = Bx x By, u1 = Bx / qx,
 * u2 = By / qy, un = u1 x u2 and the panel's inclusive 1-based pixel rectangle. Device pointers. */
#define XI_PANELS_INLINE 4         /* panel records a detector may carry inline (no device copy) */
typedef struct {
    int n_panels;
    const double *panels;           /* (n_panels, XI_PANEL_F64); NULL: the records are in panel_inline */
    int segmented;                  /* panel rectangles bound the hits; pixel_to_lab looks the panel up in segmap */
    const int16_t *segmap;          /* (seg_ny, seg_nx) panel of each pixel, -1 in gaps */
    int seg_nx, seg_ny;
    const double *geo_x, *geo_y;    /* (geo_ny, geo_nx) distortion tables (pixels); NULL: none */
    int geo_nx, geo_ny;
    int parallax;                   /* thick-sensor parallax (tsens > 0 and mu > 0) */
    double tsens, mu;
    double orgx, orgy, qx, qy, distance;
    double ed1[3], ed2[3], ed3[3];  /* detector axes as given, ed3 = ed1 x ed2 (single-panel lab map) */
    double beam[3];                 /* incident beam direction as given (Lorentz factor) */
    double pol_n[3], pol_main[3];   /* polarisation plane normal and its in-plane partner (lp_factor) */
    double pol_f;                   /* polarisation fraction */
    double nx, ny;                  /* detector size in pixels (acceptance test, regions) */
    double panel_inline[XI_PANELS_INLINE * XI_PANEL_F64];   /* used when panels is NULL (n_panels <= 4) */
} XiPlanDetector;

/* Predictions of one phi block (xpg/geometry.py:468-545 and the acceptance test of xpg/integrate.py:101-122). */
typedef struct {
    double astar[9];                /* A* row-major (columns a*, b*, c*): p = A* h */
    int hmax[3];                    /* generated grid: |h| <= hmax[0], |k| <= hmax[1], |l| <= hmax[2] */
    double q2_max, q2_min;          /* keep q2_min < |p|^2 <= q2_max (1 / dmin^2, 1 / dmax^2) */
    int centring;                   /* lattice centring letter: 'P' (none), 'C', 'A', 'B', 'I', 'F', 'R' */
    const int32_t *hkl;             /* explicit Miller indices (n_hkl, 3) instead of the grid; NULL: grid */
    int64_t n_hkl;
    double axis[3];                 /* rotation axis as given */
    double rot_K[9], rot_kk[9];     /* R(phi) = cos I + sin K + (1 - cos) kk of the unit axis */
    double s0[3];                   /* incident wave vector */
    double phi_lo, phi_hi;          /* accepted spindle angles [lo, hi) in degrees */
    double phi0, osc, z_shift;      /* z = (phi - phi0) / osc + z_shift */
    double deg, rad;                /* 180 / pi and pi / 180 as the host rounds them */
    double acc_s0[3], acc_axis[3];  /* first block's s0 and axis: zeta_k of the acceptance test */
    double min_zeta;                /* |zeta_k| >= min_zeta */
    double x_hi, y_hi;              /* 0.5 <= x < x_hi, 0.5 <= y < y_hi (first block's detector + 0.5) */
    double z_lo, z_hi;              /* z_lo <= z < z_hi */
    int block, lattice;             /* written to every row */
} XiPredict;

/* Prediction rows (device, capacity rows each). */
typedef struct {
    int32_t *hkl;                   /* (cap, 3) */
    double *phi, *S, *x, *y, *z, *zeta, *polarization, *zeta_k;     /* S: (cap, 3) */
    int32_t *block, *lattice;
} XiPredictOut;

/* Device workspace of xi_predict_count / xi_predict_write (bytes). */
size_t xi_predict_workspace(const XiPredict *P);
/* Counts the block's predictions (synchronises the stream; *n_rows on the host). The workspace keeps the counts for
 * the write that follows. */
int xi_predict_count(const XiPredict *P, const XiPlanDetector *det, void *ws, size_t ws_bytes, int64_t *n_rows,
                     void *stream);
/* Writes the block's predictions (the count call must precede it with the same arguments) into rows [0, n_rows)
 * of out; fails with XI_E_LIMIT when n_rows > cap. */
int xi_predict_write(const XiPredict *P, const XiPlanDetector *det, void *ws, size_t ws_bytes, const XiPredictOut *out,
                     int64_t cap, void *stream);

/* Shoebox rules per prediction (xpg/integrate.py:233-285 and :288-291): depth, phi binning, coverage, side,
 * super-pixels, origin, neighbour-ellipsoid widths, region, frame range. */
typedef struct {
    int64_t n;
    const double *x, *y, *z, *zeta_k;
    double sigma_m;                 /* model sigma_M (deg) */
    double abs_osc;                 /* |osc| of the first block (deg) */
    double osc2_12;                 /* osc^2 / 12 */
    double rsd_box;                 /* radians(sigma_D * widen): box side */
    double rsd;                     /* radians(sigma_D): neighbour ellipsoids */
    double qmin;                    /* min(qx, qy) */
    int box;                        /* global box side */
    int box_fixed;                  /* model.box_xy: every side is box, no super-pixels */
    int n_xyb;
    int xyb[16];                    /* side buckets below box, then box */
    int f_first, f_last;            /* frame numbers of the run */
    int n_regions_xy;
} XiBoxRules;

typedef struct {
    int32_t *iz0, *dz, *fb, *Dz, *bx, *pxs, *ix0, *iy0, *region, *zstart, *zend;
    uint8_t *flags;                 /* bit 0 wide, bit 1 truncated, bit 2 kept (a depth bucket exists) */
    float *coverage;
    double *sx_px, *sz_f;           /* neighbour-ellipsoid widths (pixels, frames) */
} XiBoxOut;

int xi_plan_boxes(const XiBoxRules *B, const XiPlanDetector *det, const XiBoxOut *out, void *stream);

/* Nearest neighbours (scipy cKDTree.query(pts, k + 1, distance_upper_bound=radius) on pts = (x / sx, y / sx,
 * z / sz), first column dropped: xpg/integrate.py:164-172): for every point its k nearest other points closer than
 * radius, by increasing distance (ties by index); missing entries j = 0, d = +inf. lo / hi bound the scaled points
 * (a cell grid over them; points outside are clamped into the edge cells, which keeps the result exact). */
#define XI_KNN_MAX 16
typedef struct {
    int64_t n;
    const double *x, *y, *z;
    double sx, sz;
    double lo[3], hi[3];
    double radius;
    int k;
} XiKnn;

size_t xi_knn_workspace(const XiKnn *q);
int xi_knn(const XiKnn *q, void *ws, size_t ws_bytes, int32_t *nbj, double *nbd, void *stream);

/* ---- Adaptation of the rocking curve (float64) -----------------------------------------------------------------
 * The per-block adaptation XPG runs in numpy on the host (xpg/integrate.py:404-461 with the grid search of
 * :1130-1154), on the block's strong reflections: their per-frame net counts fz (zero beyond each box's depth). */
typedef struct {
    int64_t n;                      /* strong reflections */
    const double *fz;               /* (n, 65) per-frame net counts */
    const int32_t *iz0;             /* (n) first frame index of each box */
    const double *phi;              /* (n) predicted spindle angle (deg) */
    const double *zeta;             /* (n) Kabsch zeta */
    double phi0, osc, z_shift;      /* frame k spans phi(k) .. phi(k + 1), phi(z) = phi0 + osc (z - z_shift) (deg) */
} XiRocking;

/* The sigma_M grid search (xpg/integrate.py:1130-1154): for each width grid[g] (deg), cost[g] = the sum over rows
 * with a positive fz total tot of tot * (fz / tot - R)^2, R the Gaussian rocking curve of that width integrated
 * over each of the 65 frames and normalised over them. */
int xi_rocking_costs(const XiRocking *q, const double *grid, int n_grid, double *cost, void *stream);

/* Normal equations of the rocking-curve mixture fit (xpg/integrate.py:437-447, the Gram form of _nnls_gram,
 * :1095-1104): gram = A^T A (21 x 21, row-major) and rhs = A^T y with A = B sqrt(tot), y = fz / tot sqrt(tot),
 * tot = max(sum fz, 1e-9), B the frame integrals of the 21 mixture components at width sm (rad). */
size_t xi_rocking_gram_workspace(const XiRocking *q);
int xi_rocking_gram(const XiRocking *q, double sm, void *ws, size_t ws_bytes, double *gram, double *rhs,
                    void *stream);

/* xi_knn without a workspace argument; it has no counterpart in XPG (whose neighbour search runs on the host).
 * For callers that cannot allocate device memory: a program binding this library through a plain C FFI beside a
 * framework that has already reserved the GPU's memory in its own pool (cudaMalloc would fail there, and
 * cudaMalloc / cudaFree can stall the whole device). The scratch memory is an array inside the library, sized for at
 * most XI_KNN_NOALLOC_MAX_POINTS points (larger calls fail with XI_E_LIMIT); bounds that would need more than
 * XI_KNN_NOALLOC_MAX_CELLS grid cells get coarser cells, with the same result. Same inputs, outputs and results as
 * xi_knn; nothing is allocated. The first call on each device looks up the array's device address: make it before
 * any stream capture. Every call on a device shares the one array, so calls that may overlap on the GPU (other
 * streams, other host threads) race and must be serialised by the caller. */
#define XI_KNN_NOALLOC_MAX_POINTS (1 << 19)
#define XI_KNN_NOALLOC_MAX_CELLS (1 << 18)
int xi_knn_noalloc(const XiKnn *q, int32_t *nbj, double *nbd, void *stream);

/* ---- Transfer encoding of uint32 frames --------------------------------------------------------------------------
 * No counterpart in XPG, which reads and decodes frames on the host (xpg/io/images.py:72-102). Raw uint32 frames
 * (Eiger-style: 0xFFFFFFFF flagged) are mostly small counts, so they cross the host-device link as one byte per
 * pixel plus exceptions and are widened back on the device, bit for bit:
 *   plane[i] = v for v < XI_PACK_ESCAPE, XI_PACK_FLAGGED for v = 0xFFFFFFFF, XI_PACK_ESCAPE otherwise;
 *   exc = (index, value) uint32 pairs of every pixel coded XI_PACK_ESCAPE, in increasing index order. */
#define XI_PACK_ESCAPE 254u
#define XI_PACK_FLAGGED 255u
#define XI_PACK_MAX_PIXELS 0xFFFFFFFFll   /* pixels per packed run (exception indices are uint32) */

/* Host function (no CUDA call): packs n pixels of host memory src into plane (n bytes) and exc (room for exc_cap
 * pairs), on `threads` host threads (0: the library's choice) of a pool kept by the library; *n_exc gets the number
 * of pairs. Fails with XI_E_LIMIT when more than exc_cap pixels need an exception (plane and exc then hold partial
 * output; send the run unpacked). Calls from several host threads are serialised. */
int xi_pack_u8(const uint32_t *src, int64_t n, uint8_t *plane, uint32_t *exc, int64_t exc_cap, int threads,
               int64_t *n_exc);

/* Widens a packed run on the device: out[i] (n uint32) from plane (n bytes) and the n_exc pairs at exc (all three
 * device memory; plane and out 16-byte aligned). */
int xi_unpack_u8(const uint8_t *plane, int64_t n, const uint32_t *exc, int64_t n_exc, uint32_t *out, void *stream);

/* A packed frame of a store of packed frames (device pointers): plane (16-byte aligned) and its exception pairs, or
 * (raw = 1) the frame's uint32 values at plane. */
typedef struct {
    const uint8_t *plane;
    const uint32_t *exc;
    int64_t n_exc;
    int raw;
} XiPackedFrame;

/* Widens n_frames packed frames of n pixels each (descriptors in device memory) into out + k * stride (out 16-byte
 * aligned, stride a multiple of 4 and >= n) in one launch. */
int xi_unpack_u8_frames(const XiPackedFrame *frames, int n_frames, int64_t n, uint32_t *out, int64_t stride,
                        void *stream);

/* ---- Bitshuffle-LZ4 frames (Eiger chunks, HDF5 filter 32008) ----------------------------------------------------
 * XPG's split of the decode (xpg/io/bslz4.py): the LZ4 stage on the host (`lz4_stage`, :35-64), the bit unshuffle on
 * the device (`unshuffle_frame_torch`, :85-121). Chunk: 8-byte big-endian uncompressed size, 4-byte big-endian block
 * size in bytes (0: 8192), per block a 4-byte big-endian compressed size and an LZ4 block; a last partial block's
 * n % 8 elements follow as they are. */

/* Host function (no CUDA call): the LZ4 stage of one chunk of esize-byte elements (2 or 4) into out (out_bytes >= the
 * chunk's uncompressed size), still bit-shuffled; *n_bytes gets that size, *block_elems the block size in elements
 * (a multiple of 8). Blocks decompress on `threads` threads of the library's pool (0: its choice). XI_E_ARG on a
 * malformed chunk (out then holds partial output). */
int xi_bslz4_lz4_stage(const uint8_t *chunk, int64_t chunk_bytes, int esize, uint8_t *out, int64_t out_bytes,
                       int threads, int64_t *n_bytes, int64_t *block_elems);

/* The bit unshuffle of a chunk's LZ4-stage output `in` (device) into n_elem uint32 values at out (device, 4-byte
 * aligned; 16-byte aligned stores when it is): 4-byte elements as they are, 2-byte elements widened with their all-ones value to 0xFFFFFFFF (the flag
 * of the uint32 frame path). */
int xi_bitunshuffle(const uint8_t *in, int64_t n_elem, int esize, int64_t block_elems, uint32_t *out, void *stream);

/* ---- Spot finding: the strong-pixel classifier -------------------------------------------------------------------
 * XPG's `make_finder(nbx, nby, signal_pixel, background_pixel, min_local, extended)` (xpg/spotfind.py:27-97): the
 * dispersion test (Kabsch 2010) on a (2 nby + 1) x (2 nbx + 1) window, then (extended) the local background
 * re-estimated over a (2 (2 nby + 1) + 1) x (2 (2 nbx + 1) + 1) window from pixels away from first-pass signal.
 * float32 frames (negative: not valid), bit for bit with the reference. */
#define XI_SPOT_MAX_HALF 8
typedef struct {
    int nbx, nby;                   /* window half-sizes, 0..XI_SPOT_MAX_HALF */
    float signal_pixel, background_pixel;
    int min_local;
    int extended;                   /* 1: the second pass */
} XiSpotParams;

/* Device scratch of an extended call (bytes). */
size_t xi_spot_workspace(int n_frames, int ny, int nx);
/* strong (uint8 0 / 1) and mean (float32) per pixel of n_frames frames of ny x nx float32 pixels (device). */
int xi_spot_strong(const float *img, int n_frames, int ny, int nx, float gain, const XiSpotParams *params,
                   uint8_t *strong, float *mean, void *ws, size_t ws_bytes, void *stream);

/* ---- INTEGRATE.HKL records ---------------------------------------------------------------------------------------
 * The data records of XPG's INTEGRATE.HKL (`write_integrate_hkl`, xpg/io/legacy.py:171-176), formatted in parallel. */
typedef struct {
    int64_t n;
    const int64_t *hkl;             /* (n, 3) */
    const double *I, *sig;          /* LP-corrected intensity and its sigma */
    const double *x, *y, *zc;       /* calculated position (zc: frame coordinate kept inside its frame) */
    const double *rlp, *peak;
    const int64_t *corr;
    const double *xo, *yo, *zo;     /* observed position (the calculated one where not observed) */
    const double *alf1, *bet1;      /* diffracted beam direction: spherical angles (deg) */
    double alf0, bet0;              /* incident beam direction */
} XiHklRows;

/* Host function: n lines " H K L I SIGMA XCAL YCAL ZCAL RLP PEAK CORR 0 XOBS YOBS ZOBS ALF0 BET0 ALF1 BET1 0.00 1"
 * (formats %.3E for I and SIGMA, %.1f positions, %.5f RLP and PEAK, %.2f angles) into out; *n_bytes gets the text's
 * size. XI_E_LIMIT when cap is smaller (then nothing is written and *n_bytes is the size needed). */
int xi_format_integrate_hkl(const XiHklRows *rows, char *out, int64_t cap, int threads, int64_t *n_bytes);

/* Copies `bytes` from page-locked host memory (cudaHostAlloc / cudaHostRegister, mapped into the device's address
 * space) to device memory with a kernel that reads the host memory over the link: unlike cudaMemcpyAsync it does not
 * queue behind the copies already waiting in the copy engine (the frame chunks), so a small upload is not delayed by
 * them. Fails with XI_E_ARG when src is not mapped page-locked host memory (checked with cudaPointerGetAttributes
 * before any launch). No counterpart in XPG (its arrays stay on the host). */
int xi_upload(const void *src, void *dst, int64_t bytes, void *stream);

/* ---- Forward-model likelihood passes ---------------------------------------------------------------------------
 * XPG's pixel-level forward integrator (xpg/forward/) models every pixel-frame of a window as a background plus
 * sum_h I_h f_h, with each reflection's fraction separable per term: f(z, y, x) = sum_t R[t, row, z] P[t, row, y, x]
 * over its box of Dz frames and b x b pixels at (iz0, iy0, ix0). Window voxels are indexed densely:
 * ((iz0 + z - f0) * ny + (iy0 + y - y0)) * nx + (ix0 + x - x0), voxels outside the window dropped
 * (WindowModel.vid, xpg/forward/model.py:381-392). These replace the Triton kernels of xpg/forward/kernels.py:34-134
 * (`scatter`, `gather`) and the eager passes WindowModel.mu / grad_ratio / grad_newton (model.py:476-577).
 * Device pointers; float32 factors and windows; int64 origins. */
typedef struct {
    int n;                          /* reflections of the chunk */
    int n_terms;                    /* separable terms T: 1 (profile) or 2 (profile and halo); at most 4 */
    int Dz, b;                      /* box frames and side */
    const float *R;                 /* (T, n, Dz) rocking-curve factors */
    const float *P;                 /* (T, n, b, b) detector-profile factors */
    const int64_t *iz0, *iy0, *ix0; /* (n) box origins: frame index, row, column (super-pixel units) */
} XiFmBoxes;

typedef struct {
    int64_t f0, nf;                 /* frames [f0, f0 + nf) (0-based frame indices) */
    int64_t y0, ny, x0, nx;         /* detector tile: rows [y0, y0 + ny), columns [x0, x0 + nx) */
} XiFmWindow;

#define XI_FM_NS_I16 0              /* counts NS as int16 (XPG's store), int32 or float32; NS < 0: no term */
#define XI_FM_NS_I32 1
#define XI_FM_NS_F32 2

/* Scatter (`kernels.scatter`, kernels.py:110-120; `WindowModel.mu`): mu[v] += I[row] * f + beta[row] over every
 * in-window voxel of every box (float atomics: the sum's order is not fixed). I, beta: (n) of the chunk's rows;
 * beta NULL: no flat term. */
int xi_fm_scatter(const XiFmBoxes *boxes, const XiFmWindow *win, const float *I, const float *beta, float *mu,
                  void *stream);

/* Gather (`kernels.gather`, kernels.py:123-134; `WindowModel.grad_ratio` / `grad_newton`) over the in-window voxels
 * with NS >= 0: mode 0: g[rows[row]] += sum f A / M; mode 1: g[rows[row]] += sum f (1 - max(NS, 0) / M) and
 * fd[rows[row]] += sum f^2 / max(M, 1e-6). rows: (n) output index of each reflection (NULL: row itself). Each
 * reflection's sums are accumulated in float64 and added once. */
int xi_fm_gather(const XiFmBoxes *boxes, const XiFmWindow *win, const int64_t *rows, const float *A, const float *M,
                 const void *NS, int ns_type, int mode, float *g, float *fd, void *stream);

/* Last error message of the forward-model passes on this thread. */
const char *xi_fm_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
