// Device planning of an integration run (include/xpgi.h, "Planning"): predictions of every Miller index of a phi
// block, the shoebox rules per prediction and the neighbour lists.
//
// XPG plans in numpy on the host; here every prediction is one thread. The arithmetic is float64 with the library's
// -fmad=false, each expression written in numpy's evaluation order (left to right, products then sums, dot products
// summed over x, y, z in turn), so the integer decisions taken on these values (boxes, buckets, frame ranges) are
// the reference's. The transcendental functions are CUDA's double-precision ones: they may differ from the host's in
// the last bit, which moves a float result by an ulp and an integer decision only when a value lies within an ulp of
// its rounding boundary.
#include <cuda_runtime.h>
#include <math.h>
#include <math_constants.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include <cub/device/device_scan.cuh>

#include "xpgi.h"
#include "xpgi_internal.h"

namespace {

constexpr int kNT = 256;                 // candidates per tile (one CTA) of the prediction kernels
constexpr int64_t kMaxCells = 1 << 22;   // cell grid of the neighbour search

// panel record offsets (XI_PANEL_F64 doubles)
enum { PR_P0 = 0, PR_BX = 3, PR_BY = 6, PR_N = 9, PR_U1 = 12, PR_U2 = 15, PR_UN = 18, PR_P0N = 21, PR_BXBX = 22,
       PR_BYBY = 23, PR_X1 = 24, PR_X2 = 25, PR_Y1 = 26, PR_Y2 = 27 };

// panel record k: device array, or the records carried in the argument itself
__device__ __forceinline__ const double* panel_rec(const XiPlanDetector& D, int k) {
    return D.panels ? D.panels + (size_t)k * XI_PANEL_F64 : D.panel_inline + k * XI_PANEL_F64;
}

__device__ __forceinline__ double dot3(const double* a, const double* b) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ double norm3(const double* a) { return sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]); }

// numpy's clip / maximum: NaN propagates
__device__ __forceinline__ double np_clip(double v, double lo, double hi) {
    if (v != v) return v;
    return v < lo ? lo : (v > hi ? hi : v);
}

__device__ __forceinline__ double np_max(double a, double b) {
    if (a != a || b != b) return a + b;
    return a > b ? a : b;
}

// numpy's float remainder: the sign of the divisor
__device__ __forceinline__ double np_mod(double a, double b) {
    double m = fmod(a, b);
    if (m != 0.0) {
        if ((b < 0.0) != (m < 0.0)) m += b;
    } else {
        m = copysign(0.0, b);
    }
    return m;
}

// float64 -> int32 as x86 converts out-of-range values (the integer indefinite)
__device__ __forceinline__ int to_i32(double v) {
    return (v >= -2147483648.0 && v < 2147483648.0) ? (int)v : INT32_MIN;
}

// bilinear distortion-table lookup (xpg/detector.py bilinear_table); NaN coordinates read the first cell and return
// NaN (the reference would index with an undefined integer)
__device__ double bilinear(const double* tab, int ny, int nx, double x, double y) {
    const double fx = np_clip(x - 1.0, 0.0, (double)nx - 1.000001);
    const double fy = np_clip(y - 1.0, 0.0, (double)ny - 1.000001);
    int ix = to_i32(floor(fx)), iy = to_i32(floor(fy));
    ix = ix < 0 ? 0 : (ix > nx - 1 ? nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy > ny - 1 ? ny - 1 : iy);
    const int ix1 = ix + 1 < nx - 1 ? ix + 1 : nx - 1;
    const int iy1 = iy + 1 < ny - 1 ? iy + 1 : ny - 1;
    const double tx = fx - (double)ix, ty = fy - (double)iy;
    const double a = tab[(size_t)iy * nx + ix] * (1.0 - tx) * (1.0 - ty);
    const double b = tab[(size_t)iy * nx + ix1] * tx * (1.0 - ty);
    const double c = tab[(size_t)iy1 * nx + ix] * (1.0 - tx) * ty;
    const double d = tab[(size_t)iy1 * nx + ix1] * tx * ty;
    return ((a + b) + c) + d;
}

// mean absorption depth of ray e projected on the panel axes (xpg/geometry.py:453-461)
__device__ void parallax_shift(const XiPlanDetector& D, const double* e, const double* u1, const double* u2,
                               const double* un, double* d1, double* d2) {
    const double cosa = np_clip(dot3(e, un), 1e-3, 1.0);
    const double L = D.tsens / cosa;
    const double muL = D.mu * L;
    const double lbar = 1.0 / D.mu - L * exp(-muL) / np_max(-expm1(-muL), 1e-12);
    *d1 = lbar * dot3(e, u1);
    *d2 = lbar * dot3(e, u2);
}

__device__ int segment_of(const XiPlanDetector& D, double x, double y) {
    if (!D.segmented) return 0;
    int ix = to_i32(floor(x - 0.5)), iy = to_i32(floor(y - 0.5));
    ix = ix < 0 ? 0 : (ix > D.seg_nx - 1 ? D.seg_nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy > D.seg_ny - 1 ? D.seg_ny - 1 : iy);
    return D.segmap[(size_t)iy * D.seg_nx + ix];
}

// lab position of the sensor entry point of detector point (x, y) (xpg/geometry.py:235-265)
__device__ void pixel_to_lab(const XiPlanDetector& D, double x, double y, double* X) {
    if (!D.segmented && !D.geo_x && !D.parallax) {
        const double a = D.qx * (x - D.orgx), b = D.qy * (y - D.orgy);
        for (int c = 0; c < 3; ++c) X[c] = (a * D.ed1[c] + b * D.ed2[c]) + D.distance * D.ed3[c];
        return;
    }
    int k = segment_of(D, x, y);
    k = k < 0 ? 0 : k;
    const double* pr = panel_rec(D, k);
    double xc = x, yc = y;
    if (D.geo_x) {
        xc = x + bilinear(D.geo_x, D.geo_ny, D.geo_nx, x, y);
        yc = y + bilinear(D.geo_y, D.geo_ny, D.geo_nx, x, y);
    }
    auto lab = [&](double a, double b) {
        for (int c = 0; c < 3; ++c) X[c] = (pr[PR_P0 + c] + (a - D.orgx) * pr[PR_BX + c]) + (b - D.orgy) * pr[PR_BY + c];
    };
    lab(xc, yc);
    if (D.parallax) {
        for (int it = 0; it < 4; ++it) {
            const double nX = norm3(X);
            const double e[3] = {X[0] / nX, X[1] / nX, X[2] / nX};
            double d1, d2;
            parallax_shift(D, e, pr + PR_U1, pr + PR_U2, pr + PR_UN, &d1, &d2);
            lab(xc - d1 / D.qx, yc - d2 / D.qy);
        }
    }
}

// detector point hit by ray S, NaN when it meets no panel (xpg/geometry.py:269-310)
__device__ void s_to_pixel(const XiPlanDetector& D, const double* S, double* px, double* py) {
    double x = CUDART_NAN, y = CUDART_NAN;
    for (int k = 0; k < D.n_panels; ++k) {
        const double* pr = panel_rec(D, k);
        const double t = pr[PR_P0N] / dot3(S, pr + PR_N);
        double P[3];
        for (int c = 0; c < 3; ++c) P[c] = t * S[c] - pr[PR_P0 + c];
        double xk = D.orgx + dot3(P, pr + PR_BX) / pr[PR_BXBX];
        double yk = D.orgy + dot3(P, pr + PR_BY) / pr[PR_BYBY];
        bool hit = isfinite(t) && t > 0.0;
        if (D.parallax) {
            const double nS = norm3(S);
            const double e[3] = {S[0] / nS, S[1] / nS, S[2] / nS};
            double d1, d2;
            parallax_shift(D, e, pr + PR_U1, pr + PR_U2, pr + PR_UN, &d1, &d2);
            xk = xk + d1 / D.qx;
            yk = yk + d2 / D.qy;
        }
        if (D.geo_x) {                          // fixed-point inversion of the distortion (xpg/detector.py:153-160)
            double xr = xk, yr = yk;
            for (int it = 0; it < 4; ++it) {
                xr = xk - bilinear(D.geo_x, D.geo_ny, D.geo_nx, xr, yr);
                yr = yk - bilinear(D.geo_y, D.geo_ny, D.geo_nx, xr, yr);
            }
            xk = xr;
            yk = yr;
        }
        if (D.segmented)
            hit = hit && xk >= pr[PR_X1] - 0.5 && xk < pr[PR_X2] + 0.5 && yk >= pr[PR_Y1] - 0.5 && yk < pr[PR_Y2] + 0.5;
        if (hit && isnan(x)) {
            x = xk;
            y = yk;
        }
    }
    *px = x;
    *py = y;
}

__device__ __forceinline__ bool centring_ok(int sym, int h, int k, int l) {
    switch (sym) {
        case 'C': return ((h + k) % 2) == 0;
        case 'A': return ((k + l) % 2) == 0;
        case 'B': return ((h + l) % 2) == 0;
        case 'I': return ((h + k + l) % 2) == 0;
        case 'F': return ((h + k) % 2) == 0 && ((k + l) % 2) == 0;
        case 'R': return ((-h + k + l) % 3) == 0;
        default: return true;
    }
}

struct PredRow {
    int h, k, l;
    double phi, S[3], x, y, z, zeta, pol, zeta_k;
};

__host__ __device__ inline int64_t grid_size(const XiPredict& P) {
    if (P.hkl) return P.n_hkl;
    return (int64_t)(2 * P.hmax[0] + 1) * (2 * P.hmax[1] + 1) * (2 * P.hmax[2] + 1);
}

// Candidate c = combo * G + g: Miller index g of the grid (or list), combo = 2 * solution + turn. True when the
// candidate is a prediction of the block that passes the acceptance test.
__device__ bool eval_candidate(const XiPredict& P, const XiPlanDetector& D, int64_t G, int64_t c, PredRow& r) {
    const int combo = (int)(c / G);
    const int64_t g = c - (int64_t)combo * G;
    int h, k, l;
    if (P.hkl) {
        h = P.hkl[3 * g];
        k = P.hkl[3 * g + 1];
        l = P.hkl[3 * g + 2];
    } else {
        const int64_t nk = 2 * P.hmax[1] + 1, nl = 2 * P.hmax[2] + 1;
        const int64_t ih = g / (nk * nl), rem = g - ih * nk * nl;
        const int64_t ik = rem / nl, il = rem - ik * nl;
        h = (int)ih - P.hmax[0];
        k = (int)ik - P.hmax[1];
        l = (int)il - P.hmax[2];
    }
    double p0[3];
    for (int i = 0; i < 3; ++i)
        p0[i] = ((double)h * P.astar[3 * i] + (double)k * P.astar[3 * i + 1]) + (double)l * P.astar[3 * i + 2];
    if (!P.hkl) {                               // generate_hkl's resolution shell and the lattice centring
        const double q2 = dot3(p0, p0);
        if (!(q2 <= P.q2_max && q2 > P.q2_min)) return false;
        if (!centring_ok(P.centring, h, k, l)) return false;
    }
    // spindle angles of the Ewald-sphere crossings (xpg/geometry.py:482-502)
    const double* m = P.axis;
    const double pm = dot3(p0, m);
    const double par[3] = {pm * m[0], pm * m[1], pm * m[2]};
    const double perp[3] = {p0[0] - par[0], p0[1] - par[1], p0[2] - par[2]};
    double mxp[3];
    cross3(m, p0, mxp);
    const double a = dot3(perp, P.s0), b = dot3(mxp, P.s0);
    const double cc = -0.5 * dot3(p0, p0) - dot3(par, P.s0);
    const double q = cc / hypot(a, b);
    if (!(fabs(q) <= 1.0)) return false;
    const double base = atan2(b, a);
    const double half = acos(np_clip(q, -1.0, 1.0));
    const double sang = (combo >> 1) == 0 ? base + half : base - half;
    double ph = sang * P.deg;
    ph = P.phi_lo + np_mod(ph - P.phi_lo, 360.0);
    const double phs = ph + ((combo & 1) ? 360.0 : 0.0);
    if (!(phs >= P.phi_lo && phs < P.phi_hi)) return false;
    // diffracted wave vector S = R(phi) p0 + s0
    const double ang = phs * P.rad;
    const double cs = cos(ang), sn = sin(ang);
    double S[3];
    for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        for (int j = 0; j < 3; ++j) {
            const double Rij = (cs * (i == j ? 1.0 : 0.0) + sn * P.rot_K[3 * i + j]) + (1.0 - cs) * P.rot_kk[3 * i + j];
            acc = acc + Rij * p0[j];
        }
        S[i] = acc + P.s0[i];
    }
    double x, y;
    s_to_pixel(D, S, &x, &y);
    if (!isfinite(x)) return false;
    const double z = (phs - P.phi0) / P.osc + P.z_shift;
    // Lorentz and polarisation factors (xpg/geometry.py:394-407)
    const double nS = norm3(S);
    const double e[3] = {S[0] / nS, S[1] / nS, S[2] / nS};
    double ce[3];
    cross3(e, D.beam, ce);
    const double zeta = dot3(ce, P.axis);
    const double em = dot3(e, D.pol_main), en = dot3(e, D.pol_n);
    const double pol = D.pol_f * (1.0 - em * em) + (1.0 - D.pol_f) * (1.0 - en * en);
    // acceptance (xpg/integrate.py:115-121): Kabsch zeta with the first block's s0 and axis, detector, frames
    double e1[3];
    cross3(S, P.acc_s0, e1);
    const double ne = np_max(norm3(e1), 1e-12);
    for (int i = 0; i < 3; ++i) e1[i] = e1[i] / ne;
    const double zk = dot3(e1, P.acc_axis);
    if (!(fabs(zk) >= P.min_zeta && x >= 0.5 && x < P.x_hi && y >= 0.5 && y < P.y_hi && z >= P.z_lo && z < P.z_hi))
        return false;
    r.h = h;
    r.k = k;
    r.l = l;
    r.phi = phs;
    for (int i = 0; i < 3; ++i) r.S[i] = S[i];
    r.x = x;
    r.y = y;
    r.z = z;
    r.zeta = zeta;
    r.pol = pol;
    r.zeta_k = zk;
    return true;
}

__global__ void __launch_bounds__(kNT) k_predict_count(XiPredict P, XiPlanDetector D, int64_t G,
                                                       long long* __restrict__ tile_count) {
    const int64_t c = (int64_t)blockIdx.x * kNT + threadIdx.x;
    PredRow r;
    const bool ok = c < 4 * G && eval_candidate(P, D, G, c, r);
    const int n = __syncthreads_count(ok);
    if (threadIdx.x == 0) tile_count[blockIdx.x] = n;
}

__global__ void __launch_bounds__(kNT) k_predict_write(XiPredict P, XiPlanDetector D, int64_t G,
                                                       const long long* __restrict__ tile_off, XiPredictOut O) {
    __shared__ int warp_off[kNT / 32];
    const int64_t c = (int64_t)blockIdx.x * kNT + threadIdx.x;
    PredRow r;
    const bool ok = c < 4 * G && eval_candidate(P, D, G, c, r);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned ball = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) warp_off[warp] = __popc(ball);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kNT / 32; ++w) {
            const int t = warp_off[w];
            warp_off[w] = s;
            s += t;
        }
    }
    __syncthreads();
    if (!ok) return;
    const int64_t o = tile_off[blockIdx.x] + warp_off[warp] + __popc(ball & ((1u << lane) - 1u));
    O.hkl[3 * o] = r.h;
    O.hkl[3 * o + 1] = r.k;
    O.hkl[3 * o + 2] = r.l;
    O.phi[o] = r.phi;
    for (int i = 0; i < 3; ++i) O.S[3 * o + i] = r.S[i];
    O.x[o] = r.x;
    O.y[o] = r.y;
    O.z[o] = r.z;
    O.zeta[o] = r.zeta;
    O.polarization[o] = r.pol;
    O.zeta_k[o] = r.zeta_k;
    O.block[o] = P.block;
    O.lattice[o] = P.lattice;
}

__global__ void k_total(const long long* __restrict__ cnt, const long long* __restrict__ off, int64_t n,
                        long long* __restrict__ total) {
    *total = n ? off[n - 1] + cnt[n - 1] : 0;
}

struct PredictWs {
    int64_t n_tiles;
    size_t cub_bytes;
    long long *count, *off, *total;
    void* cub;
    size_t bytes;
};

PredictWs predict_ws(const XiPredict* P, void* base) {
    PredictWs w{};
    const int64_t G = grid_size(*P);
    w.n_tiles = (4 * G + kNT - 1) / kNT;
    const int64_t nt = w.n_tiles > 0 ? w.n_tiles : 1;
    cub::DeviceScan::ExclusiveSum(nullptr, w.cub_bytes, (long long*)nullptr, (long long*)nullptr, (int)nt);
    char* p = static_cast<char*>(base);
    size_t o = 0;
    auto take = [&](size_t b) {
        void* q = p ? p + o : nullptr;
        o += (b + 255) / 256 * 256;
        return q;
    };
    w.count = (long long*)take(sizeof(long long) * nt);
    w.off = (long long*)take(sizeof(long long) * nt);
    w.total = (long long*)take(sizeof(long long));
    w.cub = take(w.cub_bytes);
    w.bytes = o;
    return w;
}

int predict_check(const XiPredict* P, const XiPlanDetector* D) {
    if (!P || !D) return xi_fail(XI_E_ARG, "predict: null argument");
    if (D->n_panels < 1 || (!D->panels && D->n_panels > XI_PANELS_INLINE))
        return xi_fail(XI_E_ARG, "predict: no detector panels");
    if (D->segmented && (!D->segmap || D->seg_nx < 1 || D->seg_ny < 1)) return xi_fail(XI_E_ARG, "predict: segmap");
    if (D->geo_x && (!D->geo_y || D->geo_nx < 1 || D->geo_ny < 1)) return xi_fail(XI_E_ARG, "predict: geo tables");
    if (P->hkl ? P->n_hkl < 0 : (P->hmax[0] < 0 || P->hmax[1] < 0 || P->hmax[2] < 0))
        return xi_fail(XI_E_ARG, "predict: negative size");
    const int64_t G = grid_size(*P);
    if (G > ((int64_t)1 << 36)) return xi_fail(XI_E_LIMIT, "predict: Miller-index grid beyond 2^36");
    if ((4 * G + kNT - 1) / kNT > INT32_MAX) return xi_fail(XI_E_LIMIT, "predict: too many tiles");
    return XI_OK;
}

// ---- shoebox rules ---------------------------------------------------------------------------------------------

__constant__ int c_dz_buckets[6] = {3, 5, 9, 17, 33, 65};

__global__ void k_plan_boxes(XiBoxRules B, XiPlanDetector D, XiBoxOut O) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n) return;
    const double x = B.x[i], y = B.y[i], zc = B.z[i], azk = fabs(B.zeta_k[i]);
    // depth: 4 sigma of the rocking curve each side; wide reflections binned by fb frames (xpg/integrate.py:233-250)
    const double sz = B.sigma_m / azk / B.abs_osc;
    int hz = (int)ceil(4.0 * sz + 0.5);
    const bool wide = hz > 32;
    int fb = 1;
    bool trunc = false;
    if (wide) {
        const double f = ceil((double)(2 * hz + 1) / 33.0);
        fb = (int)(f < 2.0 ? 2.0 : (f > 8.0 ? 8.0 : f));
        const double hb = ceil(4.0 * sz / (double)fb + 0.5);
        hz = (int)hb < 16 ? (int)hb : 16;
        trunc = hb > 16.0;
    }
    const int iz_c = (int)floor(zc - (double)(fb - 1) / 2.0);
    const int iz0 = iz_c - hz * fb;
    const int dz = 2 * hz + 1;
    int Dz = -1;
    for (int q = 0; q < 6; ++q)
        if (c_dz_buckets[q] >= dz) {
            Dz = c_dz_buckets[q];
            break;
        }
    float cov = 1.0f;
    if (trunc) {
        const double s2 = sqrt(2.0) * sz;
        const double v = 0.5 * (erf(((double)(iz0 + dz * fb) - zc) / s2) - erf(((double)iz0 - zc) / s2));
        cov = (float)np_clip(v, 0.0, 1.0);
    }
    // side from the local footprint of sigma_D, super-pixels, origin (xpg/integrate.py:263-285)
    double X[3];
    pixel_to_lab(D, x, y, X);
    const double Lr = norm3(X);
    int bx = B.box, pxs = 1;
    if (!B.box_fixed) {
        const double cosr = fabs(dot3(X, D.ed3)) / Lr;
        double spx = Lr * B.rsd_box / B.qmin / np_max(cosr, 0.4);
        spx = sqrt(spx * spx + 1.0 / 12.0);
        auto side = [&](double need_f) {
            const int need = 2 * max((int)ceil(need_f) + 1, 2) + 1;
            int q = 0;
            while (q < B.n_xyb && B.xyb[q] < need) ++q;
            return B.xyb[q < B.n_xyb ? q : B.n_xyb - 1];
        };
        bx = side(5.0 * spx);
        const double fp = floor(spx / 2.5);
        pxs = (int)(fp < 1.0 ? 1.0 : (fp > 4.0 ? 4.0 : fp));
        if (pxs > 1) bx = side(5.0 * spx / (double)pxs);
    }
    const int halfs = bx / 2;
    auto floordiv = [](int a, int b) { const int q = a / b; return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q; };
    const int ix0 = floordiv((int)floor(x - 1.0 + 0.5), pxs) - halfs;
    const int iy0 = floordiv((int)floor(y - 1.0 + 0.5), pxs) - halfs;
    // neighbour ellipsoids (xpg/integrate.py:287-290)
    const double sx_px = np_max(Lr * B.rsd / D.qx, 0.5) * 3.0;
    const double szr = B.sigma_m / azk;
    const double sz_f = sqrt(szr * szr + B.osc2_12) / B.abs_osc * 3.0;
    // regions (xpg/integrate.py:316-318)
    const int nr = B.n_regions_xy;
    int rx = to_i32(x / D.nx * (double)nr), ry = to_i32(y / D.ny * (double)nr);
    rx = rx < 0 ? 0 : (rx > nr - 1 ? nr - 1 : rx);
    ry = ry < 0 ? 0 : (ry > nr - 1 ? nr - 1 : ry);
    O.iz0[i] = iz0;
    O.dz[i] = dz;
    O.fb[i] = fb;
    O.Dz[i] = Dz;
    O.bx[i] = bx;
    O.pxs[i] = pxs;
    O.ix0[i] = ix0;
    O.iy0[i] = iy0;
    O.region[i] = ry * nr + rx;
    O.zstart[i] = iz0 > B.f_first - 1 ? iz0 : B.f_first - 1;
    O.zend[i] = iz0 + dz * fb - 1 < B.f_last - 1 ? iz0 + dz * fb - 1 : B.f_last - 1;
    O.flags[i] = (uint8_t)((wide ? 1 : 0) | (trunc ? 2 : 0) | (Dz > 0 ? 4 : 0));
    O.coverage[i] = cov;
    O.sx_px[i] = sx_px;
    O.sz_f[i] = sz_f;
}

// ---- neighbour search -------------------------------------------------------------------------------------------

struct KnnGrid {
    double cs;
    int dims[3];
    int64_t n_cells;
};

bool knn_grid(const XiKnn* q, KnnGrid* g, int64_t max_cells = kMaxCells) {
    if (!(q->radius > 0.0) || !isfinite(q->radius)) return false;
    double ext[3];
    for (int a = 0; a < 3; ++a) {
        ext[a] = q->hi[a] - q->lo[a];
        if (!isfinite(ext[a]) || ext[a] < 0.0) return false;
    }
    double cs = q->radius * (1.0 + 1e-9);      // points closer than radius lie in the same or adjacent cells
    for (int it = 0; it < 64; ++it) {
        int64_t n = 1;
        bool over = false;
        for (int a = 0; a < 3; ++a) {
            const double d = ceil(ext[a] / cs);
            if (d > 1e9) over = true;
            g->dims[a] = d < 1.0 ? 1 : (int)(d > 1e9 ? 1e9 : d);
            n *= g->dims[a];
            if (n > max_cells) over = true;
        }
        if (!over) {
            g->cs = cs;
            g->n_cells = n;
            return true;
        }
        cs *= 1.5;
    }
    return false;
}

struct KnnWs {
    int *count, *start, *fill, *cell_of, *sidx;
    double* spts;
    void* cub;
    size_t cub_bytes, bytes;
};

KnnWs knn_ws(const XiKnn* q, const KnnGrid& g, void* base) {
    KnnWs w{};
    cub::DeviceScan::ExclusiveSum(nullptr, w.cub_bytes, (int*)nullptr, (int*)nullptr, (int)g.n_cells);
    char* p = static_cast<char*>(base);
    size_t o = 0;
    auto take = [&](size_t b) {
        void* r = p ? p + o : nullptr;
        o += (b + 255) / 256 * 256;
        return r;
    };
    const size_t n = (size_t)(q->n > 0 ? q->n : 1);
    w.count = (int*)take(sizeof(int) * g.n_cells);
    w.start = (int*)take(sizeof(int) * g.n_cells);
    w.fill = (int*)take(sizeof(int) * g.n_cells);
    w.cell_of = (int*)take(sizeof(int) * n);
    w.sidx = (int*)take(sizeof(int) * n);
    w.spts = (double*)take(sizeof(double) * 3 * n);
    w.cub = take(w.cub_bytes);
    w.bytes = o;
    return w;
}

__global__ void k_zero2(int* __restrict__ a, int* __restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        a[i] = 0;
        b[i] = 0;
    }
}

__device__ __forceinline__ int cell_axis(double v, double lo, double cs, int dim) {
    const double f = floor((v - lo) / cs);
    if (!(f >= 0.0)) return 0;                  // NaN too
    return f >= (double)(dim - 1) ? dim - 1 : (int)f;
}

__global__ void k_knn_bin(XiKnn q, KnnGrid g, int* __restrict__ count, int* __restrict__ cell_of) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    const double p[3] = {q.x[i] / q.sx, q.y[i] / q.sx, q.z[i] / q.sz};
    int c = 0;
    for (int a = 2; a >= 0; --a) c = c * g.dims[a] + cell_axis(p[a], q.lo[a], g.cs, g.dims[a]);
    cell_of[i] = c;
    atomicAdd(&count[c], 1);
}

__global__ void k_knn_scatter(XiKnn q, const int* __restrict__ cell_of, const int* __restrict__ start,
                              int* __restrict__ fill, double* __restrict__ spts, int* __restrict__ sidx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    const int c = cell_of[i];
    const int pos = start[c] + atomicAdd(&fill[c], 1);
    spts[3 * (size_t)pos] = q.x[i] / q.sx;
    spts[3 * (size_t)pos + 1] = q.y[i] / q.sx;
    spts[3 * (size_t)pos + 2] = q.z[i] / q.sz;
    sidx[pos] = (int)i;
}

__global__ void k_knn_query(XiKnn q, KnnGrid g, const int* __restrict__ cell_of, const int* __restrict__ start,
                            const int* __restrict__ count, const double* __restrict__ spts,
                            const int* __restrict__ sidx, int32_t* __restrict__ nbj, double* __restrict__ nbd) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q.n) return;
    const int k1 = q.k + 1;
    double bd[XI_KNN_MAX + 1];
    int bj[XI_KNN_MAX + 1];
    for (int s = 0; s < k1; ++s) {
        bd[s] = CUDART_INF;
        bj[s] = INT32_MAX;
    }
    const double p[3] = {q.x[i] / q.sx, q.y[i] / q.sx, q.z[i] / q.sz};
    const double r2 = q.radius * q.radius;
    int c = cell_of[i];
    const int cx = c % g.dims[0];
    c /= g.dims[0];
    const int cy = c % g.dims[1];
    const int cz = c / g.dims[1];
    for (int zz = cz - 1; zz <= cz + 1; ++zz) {
        if (zz < 0 || zz >= g.dims[2]) continue;
        for (int yy = cy - 1; yy <= cy + 1; ++yy) {
            if (yy < 0 || yy >= g.dims[1]) continue;
            for (int xx = cx - 1; xx <= cx + 1; ++xx) {
                if (xx < 0 || xx >= g.dims[0]) continue;
                const int cell = (zz * g.dims[1] + yy) * g.dims[0] + xx;
                const int a = start[cell], e = a + count[cell];
                for (int t = a; t < e; ++t) {
                    const double dx = p[0] - spts[3 * (size_t)t];
                    const double dy = p[1] - spts[3 * (size_t)t + 1];
                    const double dz = p[2] - spts[3 * (size_t)t + 2];
                    const double d2 = (dx * dx + dy * dy) + dz * dz;
                    if (!(d2 < r2)) continue;
                    const int j = sidx[t];
                    auto before = [&](double da, int ja, double db, int jb) {
                        return da < db || (da == db && ja < jb);
                    };
                    if (!before(d2, j, bd[k1 - 1], bj[k1 - 1])) continue;
                    int s = k1 - 1;
                    while (s > 0 && before(d2, j, bd[s - 1], bj[s - 1])) {
                        bd[s] = bd[s - 1];
                        bj[s] = bj[s - 1];
                        --s;
                    }
                    bd[s] = d2;
                    bj[s] = j;
                }
            }
        }
    }
    for (int s = 1; s < k1; ++s) {
        const bool has = bd[s] < CUDART_INF;
        nbj[(size_t)i * q.k + (s - 1)] = has ? bj[s] : 0;
        nbd[(size_t)i * q.k + (s - 1)] = has ? sqrt(bd[s]) : CUDART_INF;
    }
}

int knn_check(const XiKnn* q, KnnGrid* g, int64_t max_cells = kMaxCells) {
    if (!q) return xi_fail(XI_E_ARG, "knn: null argument");
    if (q->n < 0 || q->k < 0) return xi_fail(XI_E_ARG, "knn: negative size");
    if (q->k > XI_KNN_MAX) return xi_fail(XI_E_LIMIT, "knn: k beyond XI_KNN_MAX");
    if (q->n >= INT32_MAX) return xi_fail(XI_E_LIMIT, "knn: more than 2^31 points");
    if (q->n && (!q->x || !q->y || !q->z)) return xi_fail(XI_E_ARG, "knn: null coordinates");
    if (!(q->sx > 0.0) || !(q->sz > 0.0)) return xi_fail(XI_E_ARG, "knn: scales must be positive");
    if (!knn_grid(q, g, max_cells)) return xi_fail(XI_E_ARG, "knn: bounds or radius not finite");
    return XI_OK;
}

}  // namespace

// ---- neighbour search in library-owned scratch memory (xi_knn_noalloc) -----------------------------------------
// The scratch of xi_knn (cell counters, sorted points, the scan's temporary storage) laid out for at most
// XI_KNN_NOALLOC_MAX_POINTS points on at most XI_KNN_NOALLOC_MAX_CELLS grid cells, in one array that every device
// loading the library holds (about 21 MB) until the process exits.
namespace {

constexpr size_t round256(size_t b) { return (b + 255) / 256 * 256; }
constexpr int64_t kNoAllocPoints = XI_KNN_NOALLOC_MAX_POINTS;
constexpr int64_t kNoAllocCells = XI_KNN_NOALLOC_MAX_CELLS;
constexpr size_t kNoAllocScanBytes = (size_t)1 << 20;
constexpr size_t kNoAllocBytes = 3 * round256(sizeof(int) * kNoAllocCells) + 2 * round256(sizeof(int) * kNoAllocPoints) +
                                 round256(3 * sizeof(double) * kNoAllocPoints) + kNoAllocScanBytes;
constexpr int kNoAllocDevices = 64;

}  // namespace

static __device__ __align__(256) unsigned char g_knn_scratch[kNoAllocBytes];

namespace {

std::mutex g_scratch_mu;
void* g_scratch_addr[kNoAllocDevices] = {};

// Device address of g_knn_scratch on the current device (host code sees only a stand-in for the array), looked up
// once per device.
int knn_scratch(void** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return xi_cuda_check("xi_knn_noalloc: current device");
    if (dev < 0 || dev >= kNoAllocDevices) return xi_fail(XI_E_LIMIT, "xi_knn_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_knn_scratch) != cudaSuccess || !p)
            return xi_cuda_check("xi_knn_noalloc: address of the scratch array");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return XI_OK;
}

}  // namespace

extern "C" {

size_t xi_predict_workspace(const XiPredict* P) {
    if (!P) return 0;
    return predict_ws(P, nullptr).bytes;
}

int xi_predict_count(const XiPredict* P, const XiPlanDetector* D, void* ws, size_t ws_bytes, int64_t* n_rows,
                     void* stream) {
    int rc = predict_check(P, D);
    if (rc) return rc;
    if (!n_rows) return xi_fail(XI_E_ARG, "xi_predict_count: null n_rows");
    PredictWs w = predict_ws(P, ws);
    if (!ws || ws_bytes < w.bytes) return xi_fail(XI_E_ARG, "xi_predict_count: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t G = grid_size(*P);
    *n_rows = 0;
    if (w.n_tiles == 0) return XI_OK;
    k_predict_count<<<(unsigned)w.n_tiles, kNT, 0, s>>>(*P, *D, G, w.count);
    size_t cb = w.cub_bytes;
    if (cub::DeviceScan::ExclusiveSum(w.cub, cb, w.count, w.off, (int)w.n_tiles, s) != cudaSuccess)
        return xi_cuda_check("xi_predict_count scan");
    k_total<<<1, 1, 0, s>>>(w.count, w.off, w.n_tiles, w.total);
    long long h = 0;
    if (cudaMemcpyAsync(&h, w.total, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return xi_cuda_check("xi_predict_count");
    *n_rows = h;
    return xi_cuda_check("xi_predict_count");
}

int xi_predict_write(const XiPredict* P, const XiPlanDetector* D, void* ws, size_t ws_bytes, const XiPredictOut* O,
                     int64_t cap, void* stream) {
    int rc = predict_check(P, D);
    if (rc) return rc;
    if (!O) return xi_fail(XI_E_ARG, "xi_predict_write: null output");
    PredictWs w = predict_ws(P, ws);
    if (!ws || ws_bytes < w.bytes) return xi_fail(XI_E_ARG, "xi_predict_write: workspace too small");
    cudaStream_t s = (cudaStream_t)stream;
    if (w.n_tiles == 0) return XI_OK;
    long long h = 0;
    if (cudaMemcpyAsync(&h, w.total, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return xi_cuda_check("xi_predict_write");
    if (h > cap) return xi_fail(XI_E_LIMIT, "xi_predict_write: more rows than the output capacity");
    if (h == 0) return XI_OK;
    if (!O->hkl || !O->phi || !O->S || !O->x || !O->y || !O->z || !O->zeta || !O->polarization || !O->zeta_k ||
        !O->block || !O->lattice)
        return xi_fail(XI_E_ARG, "xi_predict_write: null output column");
    k_predict_write<<<(unsigned)w.n_tiles, kNT, 0, s>>>(*P, *D, grid_size(*P), w.off, *O);
    return xi_cuda_check("xi_predict_write");
}

int xi_plan_boxes(const XiBoxRules* B, const XiPlanDetector* D, const XiBoxOut* O, void* stream) {
    if (!B || !D || !O) return xi_fail(XI_E_ARG, "xi_plan_boxes: null argument");
    if (B->n < 0) return xi_fail(XI_E_ARG, "xi_plan_boxes: negative size");
    if (B->n_xyb < 1 || B->n_xyb > 16) return xi_fail(XI_E_ARG, "xi_plan_boxes: side buckets");
    if (B->n_regions_xy < 1) return xi_fail(XI_E_ARG, "xi_plan_boxes: regions");
    if (D->n_panels < 1 || (!D->panels && D->n_panels > XI_PANELS_INLINE))
        return xi_fail(XI_E_ARG, "xi_plan_boxes: no detector panels");
    if (D->segmented && !D->segmap) return xi_fail(XI_E_ARG, "xi_plan_boxes: segmap");
    if (B->n == 0) return XI_OK;
    const unsigned nb = (unsigned)((B->n + 255) / 256);
    k_plan_boxes<<<nb, 256, 0, (cudaStream_t)stream>>>(*B, *D, *O);
    return xi_cuda_check("xi_plan_boxes");
}

size_t xi_knn_workspace(const XiKnn* q) {
    KnnGrid g;
    if (!q || !knn_grid(q, &g)) return 0;
    return knn_ws(q, g, nullptr).bytes;
}

int xi_knn(const XiKnn* q, void* ws, size_t ws_bytes, int32_t* nbj, double* nbd, void* stream) {
    KnnGrid g;
    int rc = knn_check(q, &g);
    if (rc) return rc;
    KnnWs w = knn_ws(q, g, ws);
    if (!ws || ws_bytes < w.bytes) return xi_fail(XI_E_ARG, "xi_knn: workspace too small");
    if (q->n == 0) return XI_OK;
    if (!nbj || !nbd) return xi_fail(XI_E_ARG, "xi_knn: null output");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned nb = (unsigned)((q->n + 255) / 256);
    // counters zeroed by a kernel: a memset could queue behind host-to-device transfers in the copy engine
    const int64_t zb = (g.n_cells + 255) / 256;
    k_zero2<<<(unsigned)(zb < 4096 ? zb : 4096), 256, 0, s>>>(w.count, w.fill, g.n_cells);
    k_knn_bin<<<nb, 256, 0, s>>>(*q, g, w.count, w.cell_of);
    size_t cb = w.cub_bytes;
    if (cub::DeviceScan::ExclusiveSum(w.cub, cb, w.count, w.start, (int)g.n_cells, s) != cudaSuccess)
        return xi_cuda_check("xi_knn scan");
    k_knn_scatter<<<nb, 256, 0, s>>>(*q, w.cell_of, w.start, w.fill, w.spts, w.sidx);
    if (q->k > 0) k_knn_query<<<nb, 256, 0, s>>>(*q, g, w.cell_of, w.start, w.count, w.spts, w.sidx, nbj, nbd);
    return xi_cuda_check("xi_knn");
}

int xi_knn_noalloc(const XiKnn* q, int32_t* nbj, double* nbd, void* stream) {
    KnnGrid g;
    int rc = knn_check(q, &g, kNoAllocCells);       // coarser cells when the bounds need more: same neighbours
    if (rc) return rc;
    if (q->n > kNoAllocPoints)
        return xi_fail(XI_E_LIMIT, "xi_knn_noalloc: more points than XI_KNN_NOALLOC_MAX_POINTS (524288); "
                                   "use xi_knn with a workspace");
    if (q->n == 0) return XI_OK;
    if (!nbj || !nbd) return xi_fail(XI_E_ARG, "xi_knn_noalloc: null output");
    void* base = nullptr;
    rc = knn_scratch(&base);
    if (rc) return rc;
    KnnWs w = knn_ws(q, g, base);
    if (w.bytes > kNoAllocBytes) return xi_fail(XI_E_LIMIT, "xi_knn_noalloc: scratch layout beyond the array");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned nb = (unsigned)((q->n + 255) / 256);
    // the array keeps the previous call's contents: the cell counters and fill cursors start from zero (zeroed by a
    // kernel, as in xi_knn: a memset could queue behind host-to-device transfers in the copy engine)
    const int64_t zb = (g.n_cells + 255) / 256;
    k_zero2<<<(unsigned)(zb < 4096 ? zb : 4096), 256, 0, s>>>(w.count, w.fill, g.n_cells);
    k_knn_bin<<<nb, 256, 0, s>>>(*q, g, w.count, w.cell_of);
    size_t cb = w.cub_bytes;
    if (cub::DeviceScan::ExclusiveSum(w.cub, cb, w.count, w.start, (int)g.n_cells, s) != cudaSuccess)
        return xi_cuda_check("xi_knn_noalloc scan");
    k_knn_scatter<<<nb, 256, 0, s>>>(*q, w.cell_of, w.start, w.fill, w.spts, w.sidx);
    if (q->k > 0) k_knn_query<<<nb, 256, 0, s>>>(*q, g, w.cell_of, w.start, w.count, w.spts, w.sidx, nbj, nbd);
    return xi_cuda_check("xi_knn_noalloc");
}

}  // extern "C"
