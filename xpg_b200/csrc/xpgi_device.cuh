// Device helpers of the integration kernels: float32 pixel geometry in a fixed operation order, 65-bit frame
// masks, block reductions.
//
// The translation unit is compiled with -fmad=false: every float expression is evaluated as written, one IEEE
// rounding per operation; fused multiply-adds appear only as explicit fmaf() calls, where XPG's CPU torch kernels
// fuse (3-vector norms, cross products and dot products of xpg/integrate_kernels.py:98-115, :234-238).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "xpgi.h"

namespace xi {

constexpr float kSqrt2 = 1.41421354f;          // float32(sqrt(2)), as the reference's float64 scalar rounds
constexpr float kFgR2 = 9.0f;                  // FG_R ** 2
constexpr float kBgR2 = 12.25f;                // BG_R ** 2
constexpr float kUmax = 4.5f;                  // N_BOX * 0.9
constexpr float kVarFloor = 1e-3f;
constexpr int kIrls = 6;

// ------------------------------------------------------------------------------------------------------------------
// 65-bit frame masks (Dz <= 65)
// ------------------------------------------------------------------------------------------------------------------
struct Mask65 {
    unsigned long long lo;
    unsigned hi;
    __device__ __forceinline__ void clear() { lo = 0ull; hi = 0u; }
    __device__ __forceinline__ void set(int z) {
        if (z < 64) lo |= (1ull << z); else hi |= (1u << (z - 64));
    }
    __device__ __forceinline__ bool get(int z) const {
        return z < 64 ? ((lo >> z) & 1ull) != 0ull : ((hi >> (z - 64)) & 1u) != 0u;
    }
};

// ------------------------------------------------------------------------------------------------------------------
// float32 vector arithmetic in the reference's order
// ------------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ float norm3(float x, float y, float z) {
    return sqrtf(fmaf(z, z, fmaf(y, y, x * x)));
}

__device__ __forceinline__ void cross3(const float a[3], const float b[3], float c[3]) {
    c[0] = fmaf(a[1], b[2], -(a[2] * b[1]));
    c[1] = fmaf(a[2], b[0], -(a[0] * b[2]));
    c[2] = fmaf(a[0], b[1], -(a[1] * b[0]));
}

__device__ __forceinline__ float dot3_fma(const float d[3], const float e[3]) {
    return fmaf(d[2], e[2], fmaf(d[1], e[1], d[0] * e[0]));
}

__device__ __forceinline__ float dot3_seq(const float d[3], const float e[3]) {
    float p0 = d[0] * e[0];
    float p1 = d[1] * e[1];
    float p2 = d[2] * e[2];
    return (p0 + p1) + p2;
}

__device__ __forceinline__ float erf32(float x) { return (float)erf((double)x); }
__device__ __forceinline__ float exp32(float x) { return (float)exp((double)x); }
__device__ __forceinline__ float expm1_32(float x) { return (float)expm1((double)x); }

// bilinear interpolation of a per-pixel table (xpg/detector.py:133-144), float32
__device__ __forceinline__ float table_bilinear(const float* tab, int nx, int ny, float x, float y) {
    float fx = fminf(fmaxf(x - 1.0f, 0.0f), (float)((double)nx - 1.000001));
    float fy = fminf(fmaxf(y - 1.0f, 0.0f), (float)((double)ny - 1.000001));
    int ix = (int)floorf(fx);
    int iy = (int)floorf(fy);
    int ix1 = min(ix + 1, nx - 1);
    int iy1 = min(iy + 1, ny - 1);
    float tx = fx - (float)ix;
    float ty = fy - (float)iy;
    float a = (tab[(size_t)iy * nx + ix] * (1.0f - tx)) * (1.0f - ty);
    float b = (tab[(size_t)iy * nx + ix1] * tx) * (1.0f - ty);
    float c = (tab[(size_t)iy1 * nx + ix] * (1.0f - tx)) * ty;
    float d = (tab[(size_t)iy1 * nx + ix1] * tx) * ty;
    return ((a + b) + c) + d;
}

// diffracted wave vector of detector point (x, y) (xpg/integrate_kernels.py:78-105)
__device__ inline void pixel_S(const XiDetector& d, float x, float y, float S[3]) {
    int k = 0;
    if (d.segmap) {
        int ix = min(max((int)floorf(x - 0.5f), 0), d.seg_nx - 1);
        int iy = min(max((int)floorf(y - 0.5f), 0), d.seg_ny - 1);
        k = max((int)d.segmap[(size_t)iy * d.seg_nx + ix], 0);
    }
    float P0[3], Bx[3], By[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        P0[c] = d.P0[3 * k + c];
        Bx[c] = d.Bx[3 * k + c];
        By[c] = d.By[3 * k + c];
    }
    float xc = x, yc = y;
    if (d.gx) {
        xc = x + table_bilinear(d.gx, d.geo_nx, d.geo_ny, x, y);
        yc = y + table_bilinear(d.gy, d.geo_nx, d.geo_ny, x, y);
    }
    float X[3];
    {
        float a = xc - d.orgx, b = yc - d.orgy;
#pragma unroll
        for (int c = 0; c < 3; ++c) X[c] = (P0[c] + a * Bx[c]) + b * By[c];
    }
    if (d.parallax) {
        float U1[3], U2[3], UN[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            U1[c] = d.U1[3 * k + c];
            U2[c] = d.U2[3 * k + c];
            UN[c] = d.UN[3 * k + c];
        }
        for (int it = 0; it < 2; ++it) {
            float n = norm3(X[0], X[1], X[2]);
            float e[3] = {X[0] / n, X[1] / n, X[2] / n};
            float cosa = fminf(fmaxf(dot3_seq(e, UN), 1e-3f), 1.0f);
            float L = d.tsens / cosa;
            float muL = d.mu * L;
            float lbar = d.inv_mu - (L * exp32(-muL)) / fmaxf(-expm1_32(-muL), 1e-12f);
            float d1 = lbar * dot3_seq(e, U1);
            float d2 = lbar * dot3_seq(e, U2);
            float a = (xc - d1 / d.qx) - d.orgx, b = (yc - d2 / d.qy) - d.orgy;
#pragma unroll
            for (int c = 0; c < 3; ++c) X[c] = (P0[c] + a * Bx[c]) + b * By[c];
        }
    }
    float den = norm3(X[0], X[1], X[2]) * d.wl;
#pragma unroll
    for (int c = 0; c < 3; ++c) S[c] = X[c] / den;
}

// Kabsch frame of a reflection (xpg/integrate_kernels.py:234-238)
__device__ inline void kabsch_frame(const float S[3], const float s0[3], const float axis[3], float e1[3],
                                    float e2[3], float* zeta) {
    float c1[3], c2[3];
    cross3(S, s0, c1);
    float n1 = norm3(c1[0], c1[1], c1[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) e1[c] = c1[c] / n1;
    cross3(S, e1, c2);
    float n2 = norm3(c2[0], c2[1], c2[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) e2[c] = c2[c] / n2;
    *zeta = dot3_seq(e1, axis);
}

// eps1, eps2 of detector point (x, y) (xpg/integrate_kernels.py:108-115)
__device__ __forceinline__ void eps12(const XiDetector& d, const float S[3], float invS, const float e1[3],
                                      const float e2[3], float x, float y, float* eps1, float* eps2) {
    float Sp[3];
    pixel_S(d, x, y, Sp);
    float dd[3] = {Sp[0] - S[0], Sp[1] - S[1], Sp[2] - S[2]};
    *eps1 = dot3_fma(dd, e1) * invS;
    *eps2 = dot3_fma(dd, e2) * invS;
}

// box column / row coordinate (xpg/integrate_kernels.py:224-230)
__device__ __forceinline__ float box_coord(int i0, int i, int pxs) {
    if (pxs > 1) {
        float s = (float)pxs;
        return (((float)i0 + (float)i) * s + (s - 1.0f) * 0.5f) + 1.0f;
    }
    return ((float)i0 + (float)i) + 1.0f;
}

// rocking-curve mixture fraction of one frame bin (xpg/integrate_kernels.py:130-141, :255-262); the 21 terms are
// summed in float64 in component order and rounded once
__device__ inline float rocking_fraction(float lo, float hi, float phi, float zeta, float sm, const float* rcw) {
    float s = sm / fmaxf(fabsf(zeta), 1e-3f);
    float sw = (s * 0.25f) * kSqrt2;
    double acc = 0.0;
    for (int k = 0; k < XI_RC_K; ++k) {
        float c = (k == XI_RC_K - 1) ? 3.5f : (float)((double)k * 0.35 + (-3.5));
        float cs = c * s;
        float a = ((hi - phi) - cs) / sw;
        float b = ((lo - phi) - cs) / sw;
        float term = (rcw[k] * 0.5f) * (erf32(a) - erf32(b));
        acc += (double)term;
    }
    return (float)acc;
}

// frame bin limits (xpg/integrate_kernels.py:256-260)
__device__ __forceinline__ void bin_limits(int iz0, float fb, int z, float frames_phi0, float osc, float* lo,
                                           float* hi) {
    float k = (float)iz0 + fb * (float)z;
    float plo = frames_phi0 + osc * k;
    float phi_ = plo + osc * fb;
    *lo = fminf(plo, phi_);
    *hi = fmaxf(plo, phi_);
}

// background template at a box pixel (xpg/integrate_kernels.py:68-75)
__device__ __forceinline__ float bkg_ref(const XiDetector& d, float x, float y) {
    if (!d.bkg) return 1.0f;
    int ix = min(max((int)rintf(x - 1.0f), 0), d.bkg_nx - 1);
    int iy = min(max((int)rintf(y - 1.0f), 0), d.bkg_ny - 1);
    return d.bkg[(size_t)iy * d.bkg_nx + ix];
}

// bilinear cell of normalised coordinates on the profile grid (xpg/integrate_kernels.py:154-166)
struct GridCell {
    bool inside;
    int i1, i2;
    float t1, t2;
};

__device__ __forceinline__ GridCell grid_cell(float u1, float u2) {
    const float gm1 = (float)(XI_GRID - 1);
    GridCell g;
    float f1 = ((u1 + kUmax) / 9.0f) * gm1;
    float f2 = ((u2 + kUmax) / 9.0f) * gm1;
    g.inside = (f1 >= 0.0f) && (f1 <= gm1) && (f2 >= 0.0f) && (f2 <= gm1);
    const float top = (float)((double)(XI_GRID - 1) - 1e-4);
    f1 = fminf(fmaxf(f1, 0.0f), top);
    f2 = fminf(fmaxf(f2, 0.0f), top);
    g.i1 = (int)floorf(f1);
    g.i2 = (int)floorf(f2);
    g.t1 = f1 - (float)g.i1;
    g.t2 = f2 - (float)g.i2;
    return g;
}

// P2(u) * J / seff^2 (xpg/integrate_kernels.py:278-285)
__device__ __forceinline__ float profile_value(const float* prof_r, float u1, float u2, float J, float seff) {
    GridCell g = grid_cell(u1, u2);
    const float* P = prof_r;
    float a = ((1.0f - g.t1) * (1.0f - g.t2)) * P[g.i2 * XI_GRID + g.i1];
    float b = (g.t1 * (1.0f - g.t2)) * P[g.i2 * XI_GRID + g.i1 + 1];
    float c = ((1.0f - g.t1) * g.t2) * P[(g.i2 + 1) * XI_GRID + g.i1];
    float e = (g.t1 * g.t2) * P[(g.i2 + 1) * XI_GRID + g.i1 + 1];
    float v = ((a + b) + c) + e;
    float jn = J / (seff * seff);
    return (g.inside ? v : 0.0f) * jn;
}

// ------------------------------------------------------------------------------------------------------------------
// bulk asynchronous copy of a contiguous global range into shared memory (TMA, no multicast), completion counted on
// an mbarrier. Addresses 16-byte aligned, size a multiple of 16 bytes.
// ------------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Waits for phase `parity` of the mbarrier; gives up after `max_tries` polls (returns false).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long max_tries) {
    for (long long t = 0; t < max_tries; ++t) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000000;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ------------------------------------------------------------------------------------------------------------------
// reductions
// ------------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum NV doubles over the block; results valid in `out` (shared) after the call for every thread.
// Deterministic: warps combine in warp order.
template <int NT, int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch /* [NT/32][NV] */, double* out) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double s = warp_sum(v[j]);
        if (lane == 0) scratch[w * NV + j] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int q = 0; q < NT / 32; ++q) s += scratch[q * NV + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

}  // namespace xi
