// B200 kernels of the shoebox integration path and their C ABI (include/xpgi.h).
//
// Work decomposition: one CTA per reflection. The CTA first maps its box pixels to the Kabsch frame (eps1/eps2,
// the pixel area J, u1/u2) in shared memory, then each thread owns whole pixel columns: the per-pixel terms stay in
// registers and the frame direction is walked with 65-bit masks (foreground frames, frames claimed by neighbours),
// so every voxel costs one coalesced 4-byte read per pass plus a handful of flops. Reductions accumulate in float64
// per thread and combine warp by warp in a fixed order: results do not depend on which other reflections share a
// launch.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include "xpgi_device.cuh"
#include "xpgi_internal.h"

using namespace xi;

namespace {

thread_local char g_err[512] = {0};

int fail(int code, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

int cuda_check(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof g_err, "%s: %s", where, cudaGetErrorString(e));
        return XI_E_CUDA;
    }
    return XI_OK;
}

constexpr float kSbOff = 3.0f;     // shoeboxes are stored as value + 3 (0 = unrecorded)

// neighbour data of a CTA: per active neighbour, squared normalised distances per column / row / frame
struct NbShared {
    int nact;
    int act[XI_MAX_K];
    int zmin[XI_MAX_K];             // frame of the smallest dz^2 of each active neighbour
};

// The per-axis terms of the active neighbours, in dynamic shared memory sized for the launch's neighbour columns
// and largest box: dx2 / dy2 (K x max_bx), dz2 (K x max_dz).
struct NbTab {
    float *dx2, *dy2, *dz2;
    int sxy, sz;
    __device__ __forceinline__ float& x2(int a, int i) const { return dx2[a * sxy + i]; }
    __device__ __forceinline__ float& y2(int a, int j) const { return dy2[a * sxy + j]; }
    __device__ __forceinline__ float* z2(int a) const { return dz2 + a * sz; }
};

__host__ __device__ inline size_t nb_bytes(int K, int max_bx, int max_dz) {
    return ((size_t)K * (2 * max_bx + max_dz) * sizeof(float) + 15) / 16 * 16;
}

__device__ __forceinline__ NbTab nb_tab(unsigned char* base, int K, int max_bx, int max_dz) {
    NbTab t;
    t.dx2 = reinterpret_cast<float*>(base);
    t.dy2 = t.dx2 + (size_t)K * max_bx;
    t.dz2 = t.dy2 + (size_t)K * max_bx;
    t.sxy = max_bx;
    t.sz = max_dz;
    return t;
}

// Neighbour columns whose ellipsoid reaches the box (the separable pre-test of xpg/integrate_kernels.py:192-203;
// skipping the others is exact) and their per-axis terms.
__device__ void neighbour_setup(const XiRows& R, int row, int Dz, int bx, const float* xs, const float* ys,
                                const float* zzs, bool skip_first, NbShared& nb, const NbTab& tb) {
    const int K = R.K;
    if (threadIdx.x < 32) {                  // warp 0: lane k tests neighbour column k, then the passing columns are
        const int k = threadIdx.x;           // listed in column order
        bool on = false;
        if (k < K && !(k == 0 && skip_first)) {
            float nx_ = R.nbx[(size_t)row * K + k], ny_ = R.nby[(size_t)row * K + k];
            float nz_ = R.nbz[(size_t)row * K + k];
            float sx = R.nbsx[(size_t)row * K + k], sz = R.nbsz[(size_t)row * K + k];
            float mx = (fminf(fmaxf(nx_, xs[0]), xs[bx - 1]) - nx_) / sx;
            float my = (fminf(fmaxf(ny_, ys[0]), ys[bx - 1]) - ny_) / sx;
            float mz = (fminf(fmaxf(nz_, zzs[0]), zzs[Dz - 1]) - nz_) / sz;
            on = (mx * mx + my * my) + mz * mz < 1.0f;
        }
        const unsigned ball = __ballot_sync(0xffffffffu, on);
        if (on) nb.act[__popc(ball & ((1u << k) - 1u))] = k;
        if (k == 0) nb.nact = __popc(ball);
    }
    __syncthreads();
    for (int a = 0; a < nb.nact; ++a) {
        const int k = nb.act[a];
        float nx_ = R.nbx[(size_t)row * K + k], ny_ = R.nby[(size_t)row * K + k];
        float nz_ = R.nbz[(size_t)row * K + k];
        float sx = R.nbsx[(size_t)row * K + k], sz = R.nbsz[(size_t)row * K + k];
        for (int i = threadIdx.x; i < bx; i += blockDim.x) {
            float dx = (xs[i] - nx_) / sx;
            float dy = (ys[i] - ny_) / sx;
            tb.x2(a, i) = dx * dx;
            tb.y2(a, i) = dy * dy;
        }
        for (int z = threadIdx.x; z < Dz; z += blockDim.x) {
            float dz = (zzs[z] - nz_) / sz;
            tb.z2(a)[z] = dz * dz;
        }
    }
    __syncthreads();
    // frame of each neighbour's smallest dz^2 (the first such frame): one warp per neighbour
    {
        const int lane = threadIdx.x & 31;
        for (int a = threadIdx.x >> 5; a < nb.nact; a += blockDim.x >> 5) {
            const float* d2 = tb.z2(a);
            float best = d2[0];
            int bz = 0;
            for (int z = lane; z < Dz; z += 32)
                if (d2[z] < best || (z < bz && d2[z] == best)) {
                    best = d2[z];
                    bz = z;
                }
            for (int o = 16; o > 0; o >>= 1) {
                const float ov = __shfl_down_sync(0xffffffffu, best, o);
                const int oz = __shfl_down_sync(0xffffffffu, bz, o);
                if (ov < best || (ov == best && oz < bz)) {
                    best = ov;
                    bz = oz;
                }
            }
            if (lane == 0) nb.zmin[a] = bz;
        }
    }
    __syncthreads();
}

// Frames of pixel (i, j) inside any active neighbour's ellipsoid: ((dx^2 + dy^2) + dz^2 < 1). dz^2 over the frames
// is unimodal (the bin centres increase, float subtraction, division and squaring are monotone), so for a given
// dx^2 + dy^2 the frames that pass form one interval around the minimum: found by two binary searches on the same
// float comparisons as a full scan.
__device__ __forceinline__ Mask65 neighbour_frames(const NbShared& nb, const NbTab& tb, int i, int j, int Dz) {
    Mask65 m;
    m.clear();
    for (int a = 0; a < nb.nact; ++a) {
        const float dxy = tb.x2(a, i) + tb.y2(a, j);
        const float* d2 = tb.z2(a);
        const int zm = nb.zmin[a];
        if (!(dxy + d2[zm] < 1.0f)) continue;
        int lo = 0, hi = zm;                 // first z in [0, zm] that passes
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (dxy + d2[mid] < 1.0f) hi = mid; else lo = mid + 1;
        }
        const int z0 = lo;
        lo = zm;
        hi = Dz - 1;                         // last z in [zm, Dz - 1] that passes
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (dxy + d2[mid] < 1.0f) lo = mid; else hi = mid - 1;
        }
        const int z1 = lo;
        // bits z0..z1
        if (z0 < 64) {
            const int e = min(z1, 63);
            const unsigned long long upto = (e == 63) ? ~0ull : ((1ull << (e + 1)) - 1ull);
            m.lo |= upto & ~((1ull << z0) - 1ull);
        }
        if (z1 >= 64) m.hi |= 1u;            // Dz <= 65: bit 64 only
    }
    return m;
}

// Per-pixel Kabsch mapping of a box into shared memory: eps1 -> e1s, eps2 -> e2s; then J (written to Jout when
// given, else kept in Js) and seff. On return e1s/e2s hold u1/u2 = eps/seff.
__device__ void box_geometry(const XiDetector& det, const float S[3], const float e1[3], const float e2[3],
                             int bx, const float* xs, const float* ys, float sd, float* e1s, float* e2s,
                             float* Jout, float* Js, float* seff_out) {
    const int P = bx * bx;
    const float invS = 1.0f / norm3(S[0], S[1], S[2]);
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const int i = p % bx, j = p / bx;
        float a, b;
        eps12(det, S, invS, e1, e2, xs[i], ys[j], &a, &b);
        e1s[p] = a;
        e2s[p] = b;
    }
    __syncthreads();
    __shared__ float s_seff;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const int i = p % bx, j = p / bx;
        float g[2][2];   // [field][axis x / y]
        const float* f[2] = {e1s, e2s};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float* F = f[q];
            // along x (columns)
            if (i == 0)
                g[q][0] = (-1.5f * F[p] + 2.0f * F[p + 1]) - 0.5f * F[p + 2];
            else if (i == bx - 1)
                g[q][0] = (0.5f * F[p - 2] - 2.0f * F[p - 1]) + 1.5f * F[p];
            else
                g[q][0] = (F[p + 1] - F[p - 1]) / 2.0f;
            // along y (rows)
            if (j == 0)
                g[q][1] = (-1.5f * F[p] + 2.0f * F[p + bx]) - 0.5f * F[p + 2 * bx];
            else if (j == bx - 1)
                g[q][1] = (0.5f * F[p - 2 * bx] - 2.0f * F[p - bx]) + 1.5f * F[p];
            else
                g[q][1] = (F[p + bx] - F[p - bx]) / 2.0f;
        }
        float J = fabsf(g[0][0] * g[1][1] - g[1][0] * g[0][1]);
        if (Jout) Jout[p] = J;
        if (Js) Js[p] = J;
        if (j == bx / 2 && i == bx / 2) {
            float psz = sqrtf(J);
            float q = psz / sd;
            s_seff = sd * sqrtf(1.0f + (q * q) / 12.0f);
        }
    }
    __syncthreads();
    const float seff = s_seff;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        e1s[p] = e1s[p] / seff;
        e2s[p] = e2s[p] / seff;
    }
    if (threadIdx.x == 0) *seff_out = seff;
    __syncthreads();
}

// ==================================================================================================================
// shared per-CTA helpers
// ==================================================================================================================

// Rocking-curve fractions of all Dz bins: the Dz x 21 mixture terms are spread over the CTA, then each bin sums its
// terms in component order in float64 (same value as rocking_fraction, computed 21x wider).
__device__ void rocking_curve_cta(int Dz, int iz0, float fb, const XiBlock& B, const float* rcw, float phi,
                                  float zeta, float* terms, float* R) {
    const float s = B.sm / fmaxf(fabsf(zeta), 1e-3f);
    const float sw = (s * 0.25f) * kSqrt2;
    for (int q = threadIdx.x; q < Dz * XI_RC_K; q += blockDim.x) {
        const int z = q / XI_RC_K, k = q % XI_RC_K;
        float lo, hi;
        bin_limits(iz0, fb, z, B.frames_phi0, B.osc, &lo, &hi);
        const float c = (k == XI_RC_K - 1) ? 3.5f : (float)((double)k * 0.35 + (-3.5));
        const float cs = c * s;
        const float a = ((hi - phi) - cs) / sw;
        const float b = ((lo - phi) - cs) / sw;
        terms[q] = (rcw[k] * 0.5f) * (erf32(a) - erf32(b));
    }
    __syncthreads();
    for (int z = threadIdx.x; z < Dz; z += blockDim.x) {
        double acc = 0.0;
        for (int k = 0; k < XI_RC_K; ++k) acc += (double)terms[z * XI_RC_K + k];
        R[z] = (float)acc;
    }
    __syncthreads();
}

// Per-pixel neighbour frame masks and background template of a box, computed once (shared memory). Frame 64's bit
// (boxes of 65 frames) goes to nbhi: one word per pixel, or (hi_bits) one bit per pixel, pixel p at bit p % 32 of
// word p / 32 (the form pass 2 uses, so that its tables fit the largest boxes).
__device__ void pixel_tables(const XiDetector& det, const NbShared& nb, const NbTab& tb, int bx, int Dz, const float* xs,
                             const float* ys, unsigned long long* nblo, unsigned* nbhi, float* brefs,
                             bool hi_bits = false) {
    const int P = bx * bx;
    if (nbhi && hi_bits) {
        for (int w = threadIdx.x; w < (P + 31) / 32; w += blockDim.x) nbhi[w] = 0u;
        __syncthreads();
    }
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const int i = p % bx, j = p / bx;
        const Mask65 m = neighbour_frames(nb, tb, i, j, Dz);
        nblo[p] = m.lo;
        if (nbhi) {
            if (!hi_bits) nbhi[p] = m.hi;
            else if (m.hi & 1u) atomicOr(&nbhi[p >> 5], 1u << (p & 31));
        }
        brefs[p] = bkg_ref(det, xs[i], ys[j]);
    }
    __syncthreads();
}

// Per-CTA shared copies of the small tables every pixel reads: the panel maps (up to 16 panels) and the rocking-curve
// weights. Returns the detector description with its panel pointers redirected to the shared copies.
constexpr int kSmemPanels = 16;
struct CtaTables {
    float pan[6][3 * kSmemPanels];
    float rcw[XI_RC_K];
};

__device__ XiDetector cta_tables(const XiDetector& det, const XiBlock& B, CtaTables& T) {
    XiDetector d = det;
    const int np = det.n_panels;
    if (np <= kSmemPanels) {
        for (int r = threadIdx.x; r < 3 * np; r += blockDim.x) {
            T.pan[0][r] = det.P0[r];
            T.pan[1][r] = det.Bx[r];
            T.pan[2][r] = det.By[r];
            T.pan[3][r] = det.U1[r];
            T.pan[4][r] = det.U2[r];
            T.pan[5][r] = det.UN[r];
        }
        d.P0 = T.pan[0];
        d.Bx = T.pan[1];
        d.By = T.pan[2];
        d.U1 = T.pan[3];
        d.U2 = T.pan[4];
        d.UN = T.pan[5];
    }
    for (int k = threadIdx.x; k < XI_RC_K; k += blockDim.x) T.rcw[k] = B.rcw[k];
    return d;
}

// Completes the staging of a shoebox in shared memory: waits for phase `parity` of the bulk copy's barrier (bounded;
// on a timeout the status word gets bit 2 and the values are copied with plain loads), or copies with plain loads
// when the row's arena offset is not 16-byte aligned. Ends with a barrier.
__device__ void stage_wait(bool tma, unsigned long long* bar, unsigned parity, float* stage, const float* sb, int V,
                           int* status) {
    bool ok = true;
    if (tma) ok = mbar_wait(bar, parity, 1ll << 24);
    if (!tma || !ok) {
        if (!ok && threadIdx.x == 0) atomicOr(status, 2);
        __syncthreads();
        for (int v = threadIdx.x; v < V; v += blockDim.x) stage[v] = sb[v];
    } else {
        // the bulk copy moved whole 16-byte units; the last 0..3 values come with plain loads (no read past the row)
        for (int v = (V & ~3) + threadIdx.x; v < V; v += blockDim.x) stage[v] = sb[v];
    }
    __syncthreads();
}

// ==================================================================================================================
// pass 1
// ==================================================================================================================
constexpr int kClipCand = 1024;     // background voxels above the lowest clip threshold kept per CTA
constexpr int kFgList = 2048;       // foreground pixels listed per CTA (pass C iterates them densely)
constexpr int kZBatch = 8;          // voxels of a pixel column loaded together (memory-level parallelism)
constexpr int kGatherBatch = 8;     // frames of a box pixel read together by the gather

// Dynamic shared memory: nblo (8P) | geometry scratch e1s/e2s (8P), then brefs (4P) + nbhi (4P) | flags (P) |
// img2 counts (P, padded to 16) | staged shoebox (4V, when STAGED).
__host__ __device__ inline size_t pass1_pix_bytes(int P) { return ((size_t)18 * P + 15) / 16 * 16; }

// resident CTAs per SM the pass kernels are compiled for (registers per thread <= 65536 / (NT * blocks))
// Pass 1 takes four 256-thread CTAs per SM (64 registers; measured 9% faster than three at 80 on the config-2 block
// and on deep config-4 boxes), pass 2 three (four makes it 5% slower: its spills cost more than the occupancy buys).
template <int NT> constexpr int min_ctas() { return NT == 256 ? 3 : (NT == 128 ? 6 : 8); }
template <int NT> constexpr int min_ctas_pass1() { return NT == 256 ? 4 : min_ctas<NT>(); }

// Pass 1 of one row, by the whole CTA. `bar`: the CTA's bulk-copy barrier (initialised once per CTA), `phase`: its
// next phase (advanced here when the row is staged by a bulk copy). The caller separates consecutive rows of a CTA
// with a barrier.
template <int NT, bool STAGED>
__device__ __forceinline__ void pass1_row(const XiDetector& det_g, const XiRows& R, const XiBlock& B,
                                          const float* __restrict__ arena, const XiPass1Out& O, int row, int max_bx,
                                          int max_dz, int* status, unsigned long long* bar, unsigned& phase) {
    extern __shared__ __align__(16) unsigned char dyn1[];
    __shared__ CtaTables T;
    __shared__ float xs[XI_MAX_BX], ys[XI_MAX_BX];
    __shared__ float fR[XI_MAX_DZ], fzz[XI_MAX_DZ], fe3[XI_MAX_DZ];
    // the rocking-curve terms (set-up) and the clip-candidate list (passes A and B) share one array
    constexpr int kScratch = kClipCand * 6 > XI_MAX_DZ * XI_RC_K * 4 ? kClipCand * 6 : XI_MAX_DZ * XI_RC_K * 4;
    __shared__ __align__(16) unsigned char scr[kScratch];
    float* terms = reinterpret_cast<float*>(scr);
    float* cand_v = reinterpret_cast<float*>(scr);
    unsigned short* cand_p = reinterpret_cast<unsigned short*>(scr + 4 * kClipCand);
    __shared__ NbShared nb;
    __shared__ float s_e1[3], s_e2[3], s_S[3], s_zeta, s_seff, s_b;
    __shared__ unsigned long long s_fgz_lo, s_rec_lo;
    __shared__ unsigned s_fgz_hi, s_rec_hi;
    __shared__ double red[NT / 32 * 16];
    __shared__ double tot[16];
    __shared__ float fzw[NT / 32][XI_MAX_DZ];
    // background voxels above the lowest possible clip threshold (the only ones the iterations can drop): cand_v,
    // cand_p above
    __shared__ int s_ncand;
    __shared__ unsigned short fgl[kFgList];
    __shared__ int s_nfgl;
    __shared__ int wcnt[NT / 32];
    __shared__ double s_base[2];

    const int Dz = R.Dz[row], bx = R.bx[row];
    if (Dz < 1 || Dz > max_dz || bx < 3 || bx > max_bx) {
        if (threadIdx.x == 0) atomicOr(status, 1);
        return;
    }
    const int P = bx * bx;
    const int Pm = max_bx * max_bx;                // the tables are laid out for the launch's largest box
    unsigned long long* nblo = reinterpret_cast<unsigned long long*>(dyn1);
    float* e1s = reinterpret_cast<float*>(dyn1 + (size_t)8 * Pm);
    float* e2s = e1s + Pm;
    float* brefs = e1s;                            // reuses the geometry scratch once u1 / u2 are out
    unsigned* nbhi = reinterpret_cast<unsigned*>(e1s + Pm);
    unsigned char* flags = dyn1 + (size_t)16 * Pm;
    unsigned char* imgn = dyn1 + (size_t)17 * Pm;   // per pixel: clean foreground-frame voxels | all-clean bit 7
    float* stage = reinterpret_cast<float*>(dyn1 + pass1_pix_bytes(Pm));
    const NbTab tb = nb_tab(dyn1 + pass1_pix_bytes(Pm) + (STAGED ? ((size_t)Pm * max_dz * 4 + 15) / 16 * 16 : 0), R.K,
                            max_bx, max_dz);
    const int pxs = R.pxs ? R.pxs[row] : 1;
    const int ix0 = R.ix0[row], iy0 = R.iy0[row], iz0 = R.iz0[row];
    const float fb = R.fb[row];
    const float phi = R.phi[row];
    const float* sb = arena + R.sb_off[row];
    const int64_t po = R.pix_off[row], fo = R.frm_off[row];
    const float gain = B.gain;
    auto voxel = [&](int z, int p) -> float {
        return STAGED ? stage[(size_t)z * P + p] : sb[(size_t)z * P + p] - R.sb_bias;
    };
    // the shoebox streams into shared memory (bulk copy) while the geometry below is computed
    const unsigned vbytes = (unsigned)(((size_t)Dz * P * sizeof(float)) & ~(size_t)15);   // whole 16-byte units
    const bool tma = STAGED && vbytes > 0 && ((reinterpret_cast<uintptr_t>(sb) & 15) == 0) &&
                     ((reinterpret_cast<uintptr_t>(stage) & 15) == 0);
    if (tma && threadIdx.x == 0) {
        mbar_expect_tx(bar, vbytes);
        bulk_copy_g2s(stage, sb, vbytes, bar);
    }

    const XiDetector det = cta_tables(det_g, B, T);
    if (threadIdx.x == 0) {
        float S[3] = {R.S[3 * row], R.S[3 * row + 1], R.S[3 * row + 2]};
        float e1[3], e2[3], zeta;
        kabsch_frame(S, B.s0, B.axis, e1, e2, &zeta);
        for (int c = 0; c < 3; ++c) { s_e1[c] = e1[c]; s_e2[c] = e2[c]; s_S[c] = S[c]; }
        s_zeta = zeta;
        s_rec_lo = 0ull; s_rec_hi = 0u;
    }
    for (int i = threadIdx.x; i < bx; i += NT) {
        xs[i] = box_coord(ix0, i, pxs);
        ys[i] = box_coord(iy0, i, pxs);
    }
    for (int z = threadIdx.x; z < Dz; z += NT) fzz[z] = (float)iz0 + fb * ((float)z + 0.5f);
    __syncthreads();
    const float zeta = s_zeta;
    rocking_curve_cta(Dz, iz0, fb, B, T.rcw, phi, zeta, terms, fR);
    for (int z = threadIdx.x; z < Dz; z += NT) {
        float lo, hi;
        bin_limits(iz0, fb, z, B.frames_phi0, B.osc, &lo, &hi);
        fe3[z] = zeta * (0.5f * (lo + hi) - phi);
    }
    {
        float e1[3] = {s_e1[0], s_e1[1], s_e1[2]}, e2[3] = {s_e2[0], s_e2[1], s_e2[2]};
        float S[3] = {s_S[0], s_S[1], s_S[2]};
        box_geometry(det, S, e1, e2, bx, xs, ys, B.sd, e1s, e2s, O.J + po, nullptr, &s_seff);
    }
    // u1 / u2 out, foreground / background-ring flags per pixel, and the foreground pixels listed in pixel order
    // (a block-wide ballot scan: the list, and so every later sum over it, is the same on every run)
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int base = 0;
        for (int q0 = 0; q0 < P; q0 += NT) {
            const int p = q0 + threadIdx.x;
            bool f = false;
            if (p < P) {
                const float u1 = e1s[p], u2 = e2s[p];
                O.u1[po + p] = u1;
                O.u2[po + p] = u2;
                const float r2 = u1 * u1 + u2 * u2;
                f = r2 <= kFgR2;
                flags[p] = (f ? 1 : 0) | (r2 >= kBgR2 ? 2 : 0);
            }
            const unsigned ball = __ballot_sync(0xffffffffu, f);
            if (lane == 0) wcnt[wid] = __popc(ball);
            __syncthreads();
            int off = base, all = 0;
            for (int w = 0; w < NT / 32; ++w) {
                off += w < wid ? wcnt[w] : 0;
                all += wcnt[w];
            }
            const int k = off + __popc(ball & ((1u << lane) - 1u));
            if (f && k < kFgList) fgl[k] = (unsigned short)p;
            base += all;
            __syncthreads();
        }
        if (threadIdx.x == 0) s_nfgl = base;
    }
    // foreground frames: R >= 1e-3 * Rmax + 1e-6 (warp 0: max by shuffles, the mask by ballots)
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        float Rmax = fR[0];
        for (int z = lane; z < Dz; z += 32) Rmax = fmaxf(Rmax, fR[z]);
        for (int o = 16; o > 0; o >>= 1) Rmax = fmaxf(Rmax, __shfl_xor_sync(0xffffffffu, Rmax, o));
        const float thr = 1e-3f * Rmax + 1e-6f;
        const unsigned w0 = __ballot_sync(0xffffffffu, lane < Dz && fR[lane] >= thr);
        const unsigned w1 = __ballot_sync(0xffffffffu, lane + 32 < Dz && fR[lane + 32] >= thr);
        const unsigned w2 = __ballot_sync(0xffffffffu, lane + 64 < Dz && fR[lane + 64] >= thr);
        if (lane == 0) {
            s_fgz_lo = (unsigned long long)w0 | ((unsigned long long)w1 << 32);
            s_fgz_hi = w2 & 1u;
        }
    }
    neighbour_setup(R, row, Dz, bx, xs, ys, fzz, false, nb, tb);     // ends with a barrier
    pixel_tables(det, nb, tb, bx, Dz, xs, ys, nblo, nbhi, brefs);
    Mask65 fgz;
    fgz.lo = s_fgz_lo;
    fgz.hi = s_fgz_hi;
    const float seff = s_seff;

    // ---- pass A: first background estimate, counts, recorded frames, the b-independent part of img2 --------
    // The clip threshold (bp + 3 sqrt(gain max(bp, 0.5))) + 1 is non-decreasing in bp = b * bref >= 0 (every
    // float operation in it is monotone), so it never falls below its value at bp = 0: background voxels at or
    // below that bound pass every iteration. They are summed here once; the others are listed for the iterations.
    // A pixel column's background counts are summed in float32 (exact for detector counts: integers whose column
    // sum stays below 2^24; a larger column is summed again in float64) and its template weight as count * bref,
    // so the float64 totals equal voxel-by-voxel float64 sums.
    if (STAGED) {
        stage_wait(tma, bar, phase, stage, sb, Dz * P, status);
        if (tma) phase ^= 1u;
    }
    const float clip_floor = (0.0f + 3.0f * sqrtf(gain * fmaxf(0.0f, 0.5f))) + 1.0f;
    if (threadIdx.x == 0) s_ncand = 0;
    int neg_bref = 0;
    for (int p = threadIdx.x; p < P; p += NT) neg_bref |= (brefs[p] < 0.0f);
    const bool use_list = !__syncthreads_or(neg_bref);
    const unsigned fgw[3] = {(unsigned)fgz.lo, (unsigned)(fgz.lo >> 32), fgz.hi};
    long long n_over = 0, n_fg_masked = 0, n_fg_nb = 0;
    {
        unsigned recw[3] = {0u, 0u, 0u};
        int t_over = 0, t_fgm = 0, t_fgnb = 0;
        double sc = 0.0, sb_ = 0.0, sc0 = 0.0, sb0 = 0.0;
        for (int p = threadIdx.x; p < P; p += NT) {
            const unsigned char fl = flags[p];
            const bool fg2 = fl & 1, ring = fl & 2;
            const float bref = brefs[p];
            const unsigned long long nl = nblo[p];
            const unsigned nbw[3] = {(unsigned)nl, (unsigned)(nl >> 32), nbhi[p]};
            float cs = 0.0f, cs0 = 0.0f, ic = 0.0f;
            int cn = 0, cn0 = 0, in_ = 0;
            bool okall = true;
#pragma unroll
            for (int w = 0; w < 3; ++w) {
                if (32 * w >= Dz) break;
                const int zn = min(32, Dz - 32 * w);
                const unsigned fw = fgw[w], nw = nbw[w];
                // per voxel only its value's tests are taken (valid, recorded, overloaded bits) and the two sums it
                // may join; the counts follow from the word's bit masks
                unsigned vm = 0u, rm = 0u, om = 0u;
                unsigned icm = fw & ~nw;                   // foreground frames not a neighbour's (shifted per batch)
                unsigned bgm = ring ? ~nw : 0u;            // background voxels not a neighbour's (shifted per batch)
                const float* col = (STAGED ? stage : sb) + (size_t)32 * w * P + p;
                for (int t0 = 0; t0 < zn; t0 += kZBatch) {
                  float vv[kZBatch];                     // independent loads in flight before any is used
#pragma unroll
                  for (int u = 0; u < kZBatch; ++u) vv[u] = t0 + u < zn ? col[(size_t)(t0 + u) * P] : 0.0f;
                  unsigned bv = 0u, br = 0u, bo = 0u;
#pragma unroll
                  for (int u = 0; u < kZBatch; ++u) {
                    if (t0 + u >= zn) break;
                    const float v = vv[u] - R.sb_bias;
                    if (STAGED) stage[(size_t)(32 * w + t0 + u) * P + p] = v;
                    const bool valid = v >= 0.0f;
                    bv |= (unsigned)valid << u;
                    br |= (unsigned)(v > -2.5f) << u;
                    bo |= (unsigned)(v == -2.0f) << u;
                    if (valid && ((icm >> u) & 1u)) ic += v;
                    if (valid && ((bgm >> u) & 1u)) {    // background (the ring excludes the foreground ellipse)
                        if (v <= clip_floor) {
                            cs0 += v;
                            ++cn0;
                        } else {
                            cs += v;
                            ++cn;
                            if (use_list) {
                                const int k = atomicAdd(&s_ncand, 1);
                                if (k < kClipCand) {
                                    cand_v[k] = v;
                                    cand_p[k] = (unsigned short)p;
                                }
                            }
                        }
                    }
                  }
                  vm |= bv << t0;
                  rm |= br << t0;
                  om |= bo << t0;
                  icm >>= kZBatch;
                  bgm >>= kZBatch;
                }
                recw[w] |= rm;
                const unsigned fgm = fg2 ? fw : 0u;     // foreground voxels of this column
                t_over += __popc(fgm & om);
                t_fgm += __popc(fgm & ~vm & rm);
                t_fgnb += __popc(fgm & nw);
                const unsigned clean_fg = fw & vm & ~nw; // foreground-frame voxels valid and not a neighbour's
                in_ += __popc(clean_fg);
                if (clean_fg != fw) okall = false;
            }
            double csd = (double)cs;
            if (cs >= 16777216.0f) {                     // float32 may have rounded: this column again in float64
                csd = 0.0;
                for (int z = 0; z < Dz; ++z) {
                    const float v = voxel(z, p);
                    const bool nbz = z < 64 ? ((nl >> z) & 1ull) : (nbw[2] & 1u);
                    if (ring && v >= 0.0f && !nbz && v > clip_floor) csd += (double)v;
                }
            }
            sc += csd + (double)cs0;
            sb_ += (double)(cn + cn0) * (double)bref;
            sc0 += (double)cs0;
            sb0 += (double)cn0 * (double)bref;
            O.img2[po + p] = ic;                         // completed with the background after pass B
            imgn[p] = (unsigned char)(in_ | (okall ? 0x80 : 0));
        }
        double a7[7] = {sc, sb_, (double)t_over, (double)t_fgm, (double)t_fgnb, sc0, sb0};
        atomicOr(&s_rec_lo, (unsigned long long)recw[0] | ((unsigned long long)recw[1] << 32));
        atomicOr(&s_rec_hi, recw[2]);
        block_sum<NT, 7>(a7, red, tot);
        if (threadIdx.x == 0) {
            s_b = (float)tot[0] / fmaxf((float)tot[1], 1e-6f);
            s_base[0] = tot[5];
            s_base[1] = tot[6];
        }
        __syncthreads();
        n_over = (long long)tot[2];
        n_fg_masked = (long long)tot[3];
        n_fg_nb = (long long)tot[4];
    }
    const bool listed = use_list && s_ncand <= kClipCand && P <= 65536;
    // ---- passes B: Poisson-aware clipped background, 4 iterations (background-ring pixels only) ---------------
    double nbg_d = 0.0;
    for (int it = 0; it < 4; ++it) {
        const float b = s_b;
        double sc = 0.0, sb_ = 0.0;
        if (listed) {
            for (int k = threadIdx.x; k < s_ncand; k += NT) {
                const float v = cand_v[k];
                const float bref = brefs[cand_p[k]];
                const float bp = b * bref;
                const float thr = (bp + 3.0f * sqrtf(gain * fmaxf(bp, 0.5f))) + 1.0f;
                if (v <= thr) {
                    sc += (double)v;
                    sb_ += (double)bref;
                }
            }
            double a2[2] = {sc, sb_};
            block_sum<NT, 2>(a2, red, tot);
            const double tc = s_base[0] + tot[0], tb = s_base[1] + tot[1];
            if (threadIdx.x == 0) s_b = (float)tc / fmaxf((float)tb, 1e-6f);
            nbg_d = tb;
            __syncthreads();
            continue;
        }
        for (int p = threadIdx.x; p < P; p += NT) {
            if (!(flags[p] & 2)) continue;          // r2 >= 12.25 also excludes the foreground ellipse
            const float bref = brefs[p];
            const float bp = b * bref;
            const float thr = (bp + 3.0f * sqrtf(gain * fmaxf(bp, 0.5f))) + 1.0f;
            Mask65 nbm;
            nbm.lo = nblo[p];
            nbm.hi = nbhi[p];
            for (int z = 0; z < Dz; ++z) {
                const float v = voxel(z, p);
                if (v >= 0.0f && !nbm.get(z) && v <= thr) {
                    sc += (double)v;
                    sb_ += (double)bref;
                }
            }
        }
        double a2[2] = {sc, sb_};
        block_sum<NT, 2>(a2, red, tot);
        if (threadIdx.x == 0) s_b = (float)tot[0] / fmaxf((float)tot[1], 1e-6f);
        nbg_d = tot[1];
        __syncthreads();
    }
    const float b = s_b;
    // ---- pass C: summation, centroid, moments, per-frame net over the listed foreground pixels; img2 ---------
    // img2 is linear in the background: each pixel's clean foreground-frame count sum (pass A) minus its count of
    // such voxels times b * bref. The foreground sums run over the pixel list (every lane a foreground pixel);
    // a column's sums are taken in float32 (<= 65 terms), then weighted by the pixel's constants and added in
    // float64.
    for (int p = threadIdx.x; p < P; p += NT) {
        const unsigned char m = imgn[p];
        O.img2[po + p] = O.img2[po + p] - (float)(m & 0x7f) * (b * brefs[p]);
        O.all_valid2[po + p] = m >> 7;
    }
    double acc[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc[q] = 0.0;
    for (int z = threadIdx.x; z < Dz; z += NT)
        for (int w = 0; w < NT / 32; ++w) fzw[w][z] = 0.0f;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nfl = s_nfgl;
    const bool fl_listed = nfl <= kFgList;
    const int n_items = fl_listed ? nfl : P;
    const int n_iter = (n_items + NT - 1) / NT;
    for (int q = 0; q < n_iter; ++q) {
        const int k = threadIdx.x + q * NT;
        int p = 0;
        bool have = false;
        if (k < n_items) {
            p = fl_listed ? (int)fgl[k] : k;
            have = fl_listed || (flags[p] & 1);
        }
        if (!__any_sync(0xffffffffu, have)) continue;      // warp-uniform: no foreground pixel in this warp
        const int i = p % bx, j = p / bx;
        float u1 = 0.f, u2 = 0.f, bref = 1.f;
        unsigned nbw[3] = {0u, 0u, 0u};
        if (have) {
            u1 = O.u1[po + p];
            u2 = O.u2[po + p];
            bref = brefs[p];
            const unsigned long long nl = nblo[p];
            nbw[0] = (unsigned)nl;
            nbw[1] = (unsigned)(nl >> 32);
            nbw[2] = nbhi[p];
        }
        const float bpix = b * bref;
        float c_n = 0.f, c_net = 0.f, c_c = 0.f, c_w = 0.f, c_wz = 0.f, c_e3 = 0.f, c_e33 = 0.f;
        int c_raw = 0;                                       // exact: <= 65 counts below 2^23 each
#pragma unroll
        for (int w = 0; w < 3; ++w) {
            if (32 * w >= Dz) break;
            const int zn = min(32, Dz - 32 * w);
            const unsigned fw = fgw[w], nw = nbw[w];
            const float* col = (STAGED ? stage : sb) + (size_t)32 * w * P + p;
            for (int t0 = 0; t0 < zn; t0 += kZBatch) {
              float vv[kZBatch];
#pragma unroll
              for (int u = 0; u < kZBatch; ++u) vv[u] = have && t0 + u < zn ? col[(size_t)(t0 + u) * P] : 0.0f;
#pragma unroll
              for (int u = 0; u < kZBatch; ++u) {
                const int t = t0 + u;
                if (t >= zn) break;
                const int z = 32 * w + t;
                float fzc = 0.0f;
                if (have) {
                    const float v = STAGED ? vv[u] : vv[u] - R.sb_bias;
                    const bool valid = v >= 0.0f;
                    const float c = valid ? v : 0.0f;
                    const bool clean = valid && !((nw >> t) & 1u);
                    const float net = c - bpix;
                    if (clean) {
                        fzc = net;
                        if ((fw >> t) & 1u) {                // fgv: foreground, valid, not a neighbour's
                            c_n += 1.0f;
                            c_net += net;
                            c_c += c;
                            c_raw += (int)c;
                            const float wpos = fmaxf(net, 0.0f);
                            c_w += wpos;
                            c_wz += wpos * fzz[z];
                            const float e3 = fe3[z];
                            c_e3 += net * e3;
                            c_e33 += net * (e3 * e3);
                        }
                    }
                }
                fzc = warp_sumf(fzc);
                if (lane == 0) fzw[wid][z] += fzc;
              }
            }
        }
        if (have && c_n > 0.0f) {
            const float x = xs[i], y = ys[j];
            const float eps1 = u1 * seff, eps2 = u2 * seff;
            const float e12 = eps1 * eps1 + eps2 * eps2;
            acc[14] += (double)c_n;
            acc[0] += (double)c_n * (double)bref;             // sfb
            acc[1] += (double)c_net;                          // isum
            acc[2] += (double)c_c;                            // vsum counts
            acc[3] += (double)c_n * (double)bpix;             // vsum0
            acc[4] += (double)c_w;                            // sw
            acc[5] += (double)c_w * (double)x;
            acc[6] += (double)c_w * (double)y;
            acc[7] += (double)c_wz;
            acc[8] += (double)c_net;                          // sws
            acc[9] += (double)c_net * (double)eps1;
            acc[10] += (double)c_net * (double)eps2;
            acc[11] += (double)c_net * (double)e12;
            acc[12] += (double)c_e3;
            acc[13] += (double)c_e33;
            acc[15] += (double)c_raw;                         // integer partial sums below 2^53: exact
        }
    }
    block_sum<NT, 16>(acc, red, tot);
    for (int z = threadIdx.x; z < Dz; z += NT) {
        float s = 0.0f;
        for (int w = 0; w < NT / 32; ++w) s += fzw[w][z];
        O.fz[fo + z] = s;
    }
    if (threadIdx.x == 0) {
        Mask65 rm;
        rm.lo = s_rec_lo;
        rm.hi = s_rec_hi;
        double fr = 0.0;
        for (int z = 0; z < Dz; ++z)
            if (rm.get(z)) fr += (double)fR[z];
        const float nbg = (float)nbg_d;
        const float sfb = (float)tot[0];
        const float tail = ((sfb * sfb) * gain) * fmaxf(b, kVarFloor) / fmaxf(nbg, 1.0f);
        const float vsum = gain * (float)tot[2] + tail;
        const float vsum0 = gain * (float)tot[3] + tail;
        const float sw = fmaxf((float)tot[4], 1e-6f);
        const float sws = fmaxf((float)tot[8], 1e-6f);
        const float mu1 = (float)tot[9] / sws, mu2 = (float)tot[10] / sws;
        const float m_d = (((float)tot[11] / sws - mu1 * mu1) - mu2 * mu2) / 2.0f;
        const float mu3 = (float)tot[12] / sws;
        const float m_m = (float)tot[13] / sws - mu3 * mu3;
        O.bg[row] = b;
        O.nbg[row] = nbg;
        O.isum[row] = (float)tot[1];
        O.vsum[row] = vsum;
        O.vsum0[row] = vsum0;
        O.xo[row] = (float)tot[5] / sw;
        O.yo[row] = (float)tot[6] / sw;
        O.zo[row] = (float)tot[7] / sw;
        O.m_d[row] = m_d;
        O.m_m[row] = m_m;
        O.frac_rec[row] = (float)fr;
        O.nfg[row] = (float)tot[14];
        O.zeta[row] = zeta;
        O.seff[row] = seff;
        O.n_over[row] = n_over;
        O.n_fg_masked[row] = n_fg_masked;
        O.n_fg_nb[row] = n_fg_nb;
        if (O.isum_raw) O.isum_raw[row] = (int64_t)tot[15];
    }
}

// Pass 1, one CTA per row of `order` (one shoebox shape group per launch).
template <int NT, bool STAGED>
__global__ void __launch_bounds__(NT, min_ctas_pass1<NT>()) k_pass1(XiDetector det_g, XiRows R, XiBlock B,
                                                              const float* __restrict__ arena, XiPass1Out O,
                                                              const int32_t* __restrict__ order, int max_bx,
                                                              int max_dz, int* status) {
    __shared__ __align__(8) unsigned long long s_bar;
    if (STAGED && threadIdx.x == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    unsigned phase = 0;
    pass1_row<NT, STAGED>(det_g, R, B, arena, O, order ? order[blockIdx.x] : blockIdx.x, max_bx, max_dz, status,
                          &s_bar, phase);
}

// A row set's description copied into the CTA's shared memory (all threads take the same branch: `cur` was read
// after a barrier); thread 0 records which set it holds once every thread has passed the test.
__device__ __forceinline__ void load_set(const XiRowSet* __restrict__ sets, int set, XiRowSet* buf, int* cur) {
    const int* src = reinterpret_cast<const int*>(sets + set);
    int* dst = reinterpret_cast<int*>(buf);
    for (int w = threadIdx.x; w < (int)(sizeof(XiRowSet) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    if (threadIdx.x == 0) *cur = set;
}

// Pass 1 over a queue of (set, row) items: resident CTAs take items in queue order until it is empty, so rows of
// any blocks and sweeps (of one size bin) share one launch with no tail between shape groups.
template <int NT, bool STAGED>
__global__ void __launch_bounds__(NT, min_ctas_pass1<NT>()) k_pass1_q(const XiRowSet* __restrict__ sets,
                                                                const int64_t* __restrict__ items, int n_items,
                                                                int max_bx, int max_dz, int max_k, int* queue,
                                                                int* status) {
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ XiRowSet s_set;
    __shared__ int s_item, s_cur;
    if (threadIdx.x == 0) {
        if (STAGED) mbar_init(&s_bar, 1);
        s_cur = -1;
    }
    unsigned phase = 0;
    for (;;) {
        __syncthreads();                 // the previous row's shared memory is free
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) return;
        const int64_t v = items[it];
        const int set = (int)(v >> 32);
        if (set != s_cur) load_set(sets, set, &s_set, &s_cur);
        if (s_set.rows.K > max_k) {          // neighbour tables are sized for max_k columns: skip, flag
            if (threadIdx.x == 0) atomicOr(status, 1);
            continue;
        }
        pass1_row<NT, STAGED>(s_set.det, s_set.rows, s_set.blk, s_set.arena, s_set.p1, (int)(v & 0xffffffffll),
                              max_bx, max_dz, status, &s_bar, phase);
    }
}

// ==================================================================================================================
// pass 2
// ==================================================================================================================
// Dynamic shared memory: nblo (8P, first the partner's eps1 / eps2) | P2s (4P) | P2ps (4P) | brefs (4P, first the
// partner's J) | nbhi (one bit per pixel, only when boxes reach frame 64, whose bit it holds) | fit list (8 x cap,
// first the rocking-curve terms) | staged net counts of the fitted voxels (4V, when STAGED).
__host__ __device__ inline size_t pass2_pix_bytes(int P, int max_dz) {
    return ((size_t)20 * P + (max_dz > 64 ? (size_t)(P + 31) / 32 * 4 : 0) + 15) / 16 * 16;
}
__host__ __device__ inline size_t pass2_list_bytes(int cap) {
    const size_t b = (size_t)8 * cap, t = (size_t)XI_MAX_DZ * XI_RC_K * sizeof(float);
    return ((b > t ? b : t) + 15) / 16 * 16;
}
__host__ __device__ inline size_t pass2_stage_offset(int P, int max_dz, int cap) {
    return pass2_pix_bytes(P, max_dz) + pass2_list_bytes(cap);
}

// Pass 2 of one row, by the whole CTA (barrier and phase as in pass1_row).
template <int NT, bool STAGED>
__device__ __forceinline__ void pass2_row(const XiDetector& det_g, const XiRows& R, const XiBlock& B,
                                          const float* __restrict__ arena, const float* __restrict__ prof,
                                          const XiPass2In& I2, const XiPass2Out& O, int row, int max_bx, int max_dz,
                                          int cap, int* status, unsigned long long* bar, unsigned& phase) {
    extern __shared__ __align__(16) unsigned char dyn2[];
    __shared__ CtaTables T;
    __shared__ float s_prof[XI_GRID * XI_GRID];
    __shared__ int s_nlist;
    __shared__ float xs[XI_MAX_BX], ys[XI_MAX_BX];
    __shared__ float fR[XI_MAX_DZ], fRp[XI_MAX_DZ], fzz[XI_MAX_DZ];
    __shared__ NbShared nb;
    __shared__ float s_e1[3], s_e2[3], s_S[3], s_zetap, s_seffp;
    __shared__ float s_I, s_Ip, s_pmax, s_ppmax;
    __shared__ unsigned long long s_fgz_lo;
    __shared__ unsigned s_fgz_hi;
    __shared__ double red[NT / 32 * 16];
    __shared__ double tot[16];
    __shared__ float fmax_w[NT / 32][2];

    const int Dz = R.Dz[row], bx = R.bx[row];
    if (Dz < 1 || Dz > max_dz || bx < 3 || bx > max_bx) {
        if (threadIdx.x == 0) atomicOr(status, 1);
        return;
    }
    const int P = bx * bx;
    const int Pm = max_bx * max_bx;
    unsigned long long* nblo = reinterpret_cast<unsigned long long*>(dyn2);
    float* e1s = reinterpret_cast<float*>(dyn2);          // partner geometry, before nblo is written
    float* e2s = e1s + Pm;
    float* P2s = reinterpret_cast<float*>(dyn2 + (size_t)8 * Pm);
    float* P2ps = P2s + Pm;
    float* brefs = P2ps + Pm;
    float* Jps = brefs;                                   // partner J, before brefs is written
    unsigned* nbhi = max_dz > 64 ? reinterpret_cast<unsigned*>(brefs + Pm) : nullptr;   // frame 64's bits
    auto hi_bit = [&](int p) -> unsigned { return nbhi ? (nbhi[p >> 5] >> (p & 31)) & 1u : 0u; };
    float* ul_v = reinterpret_cast<float*>(dyn2 + pass2_pix_bytes(Pm, max_dz));      // fit list: net counts
    float* terms = ul_v;                                  // rocking-curve terms, before the fit list is written
    unsigned* ul_i = reinterpret_cast<unsigned*>(ul_v + cap);                 // fit list: z << 16 | pixel
    float* stage = reinterpret_cast<float*>(dyn2 + pass2_stage_offset(Pm, max_dz, cap));   // 16-byte aligned
    const NbTab tb = nb_tab(dyn2 + pass2_stage_offset(Pm, max_dz, cap) + (STAGED ? ((size_t)Pm * max_dz * 4 + 15) / 16 * 16 : 0),
                            R.K, max_bx, max_dz);
    const int pxs = R.pxs ? R.pxs[row] : 1;
    const int ix0 = R.ix0[row], iy0 = R.iy0[row], iz0 = R.iz0[row];
    const float fb = R.fb[row];
    const float phi = R.phi[row];
    const bool has_p = R.has_p[row] > 0.5f;
    const float hp = R.has_p[row];
    const float* sb = arena + R.sb_off[row];
    const int64_t po = R.pix_off[row];
    const float gain = B.gain;
    const float zeta = I2.zeta[row], seff = I2.seff[row];
    const float bg = I2.bg[row], nbgv = I2.nbg[row];
    const float* prof_g = prof + (size_t)R.region[row] * XI_GRID * XI_GRID;
    for (int q = threadIdx.x; q < XI_GRID * XI_GRID; q += NT) s_prof[q] = prof_g[q];
    const float* prof_r = s_prof;
    const XiDetector det = cta_tables(det_g, B, T);
    const unsigned vbytes = (unsigned)(((size_t)Dz * P * sizeof(float)) & ~(size_t)15);   // whole 16-byte units
    const bool tma = STAGED && vbytes > 0 && ((reinterpret_cast<uintptr_t>(sb) & 15) == 0) &&
                     ((reinterpret_cast<uintptr_t>(stage) & 15) == 0);
    if (tma && threadIdx.x == 0) {
        mbar_expect_tx(bar, vbytes);
        bulk_copy_g2s(stage, sb, vbytes, bar);
    }

    for (int i = threadIdx.x; i < bx; i += NT) {
        xs[i] = box_coord(ix0, i, pxs);
        ys[i] = box_coord(iy0, i, pxs);
    }
    for (int z = threadIdx.x; z < Dz; z += NT) fzz[z] = (float)iz0 + fb * ((float)z + 0.5f);
    if (threadIdx.x == 0 && has_p) {
        float S[3] = {R.pS[3 * row], R.pS[3 * row + 1], R.pS[3 * row + 2]};
        float e1[3], e2[3], zp;
        kabsch_frame(S, B.s0, B.axis, e1, e2, &zp);
        for (int c = 0; c < 3; ++c) { s_e1[c] = e1[c]; s_e2[c] = e2[c]; s_S[c] = S[c]; }
        s_zetap = zp;
    }
    __syncthreads();
    rocking_curve_cta(Dz, iz0, fb, B, T.rcw, phi, zeta, terms, fR);
    if (has_p) {
        rocking_curve_cta(Dz, iz0, fb, B, T.rcw, R.pphi[row], s_zetap, terms, fRp);
        float e1[3] = {s_e1[0], s_e1[1], s_e1[2]}, e2[3] = {s_e2[0], s_e2[1], s_e2[2]};
        float S[3] = {s_S[0], s_S[1], s_S[2]};
        box_geometry(det, S, e1, e2, bx, xs, ys, B.sd, e1s, e2s, nullptr, Jps, &s_seffp);
    } else {
        for (int z = threadIdx.x; z < Dz; z += NT) fRp[z] = 0.0f;
        __syncthreads();
    }
    // per-pixel profile planes; the profile maxima follow from them (f32 products are monotone in R)
    float Rmax = fR[0], Rpmax = fRp[0];
    for (int z = 1; z < Dz; ++z) {
        Rmax = fmaxf(Rmax, fR[z]);
        Rpmax = fmaxf(Rpmax, fRp[z]);
    }
    float pm_t = 0.0f, ppm_t = 0.0f;
    for (int p = threadIdx.x; p < P; p += NT) {
        const float J = I2.J[po + p];
        const float v = profile_value(prof_r, I2.u1[po + p], I2.u2[po + p], J, seff);
        P2s[p] = v;
        pm_t = fmaxf(pm_t, v * Rmax);
        if (has_p) {
            const float vp = profile_value(prof_r, e1s[p], e2s[p], Jps[p], s_seffp);
            P2ps[p] = vp;
            ppm_t = fmaxf(ppm_t, (vp * Rpmax) * hp);
        } else {
            P2ps[p] = 0.0f;
        }
    }
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int o = 16; o > 0; o >>= 1) {
            pm_t = fmaxf(pm_t, __shfl_down_sync(0xffffffffu, pm_t, o));
            ppm_t = fmaxf(ppm_t, __shfl_down_sync(0xffffffffu, ppm_t, o));
        }
        if (lane == 0) { fmax_w[wid][0] = pm_t; fmax_w[wid][1] = ppm_t; }
        __syncthreads();
        if (threadIdx.x == 0) {
            float a = 0.0f, c = 0.0f;
            for (int w = 0; w < NT / 32; ++w) { a = fmaxf(a, fmax_w[w][0]); c = fmaxf(c, fmax_w[w][1]); }
            s_pmax = a;
            s_ppmax = c;
            float thr = 1e-3f * Rmax + 1e-6f;
            Mask65 m;
            m.clear();
            for (int z = 0; z < Dz; ++z)
                if (fR[z] >= thr) m.set(z);
            s_fgz_lo = m.lo;
            s_fgz_hi = m.hi;
        }
        __syncthreads();
    }
    neighbour_setup(R, row, Dz, bx, xs, ys, fzz, has_p, nb, tb);     // ends with a barrier (partner scratch free)
    pixel_tables(det, nb, tb, bx, Dz, xs, ys, nblo, nbhi, brefs, true);
    const float pthr = 0.01f * s_pmax;
    const float ppthr = 0.01f * fmaxf(s_ppmax, 1e-12f);

    // ---- pass U: the profile sums, the fit mask, the fit sums that do not depend on I. The fitted voxels (net count
    // and packed frame / pixel index) are compacted into a shared-memory list that every later pass iterates
    // densely; when the list overflows, the later passes fall back to scanning the box (staged copy or global).
    Mask65 fgz;
    fgz.lo = s_fgz_lo;
    fgz.hi = s_fgz_hi;
    if (STAGED) {
        stage_wait(tma, bar, phase, stage, sb, Dz * P, status);
        if (tma) phase ^= 1u;
    }
    if (threadIdx.x == 0) s_nlist = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    // frame sums of the rocking curve: a pixel's profile total is P2 * sum_z R (all frames) and its foreground
    // share P2 * sum_{z in fgz} R, both taken per pixel in float64; p_valid subtracts the frames a pixel loses
    // (masked voxels, neighbours), summed per column
    __shared__ double s_rsum[2];
    if (threadIdx.x == 0) {
        double ra = 0.0, rf = 0.0;
        for (int z = 0; z < Dz; ++z) {
            ra += (double)fR[z];
            if (fgz.get(z)) rf += (double)fR[z];
        }
        s_rsum[0] = ra;
        s_rsum[1] = rf;
    }
    __syncthreads();
    const double r_all = s_rsum[0], r_fg = s_rsum[1];
    {
        double a8[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // s_net, s_w, p_total, p_valid, p_fgn, a110, C0, nuse
        const int n_iter = (P + NT - 1) / NT;
        for (int q = 0; q < n_iter; ++q) {
            const int p = threadIdx.x + q * NT;
            const bool have = p < P;
            float bref = 1.0f, P2 = 0.0f, P2p = 0.0f;
            bool fg2 = false;
            unsigned nbw[3] = {0u, 0u, 0u};
            if (have) {
                bref = brefs[p];
                P2 = P2s[p];
                P2p = P2ps[p];
                const float u1 = I2.u1[po + p], u2 = I2.u2[po + p];
                fg2 = (u1 * u1 + u2 * u2) <= kFgR2;
                const unsigned long long nl = nblo[p];
                nbw[0] = (unsigned)nl;
                nbw[1] = (unsigned)(nl >> 32);
                nbw[2] = hi_bit(p);
            }
            const float bpix = bg * bref;
            const float iv0 = __frcp_rn(gain * fmaxf(bpix, kVarFloor));
            unsigned umw[3] = {0u, 0u, 0u};      // frames of this pixel that enter the fit
            float lost = 0.0f;                   // rocking-curve weight of the frames this pixel loses
#pragma unroll
            for (int w = 0; w < 3; ++w) {
                if (32 * w >= Dz) break;
                const int zn = min(32, Dz - 32 * w);
                const unsigned nw = nbw[w];
                const float* col = (STAGED ? stage : sb) + (size_t)32 * w * P + p;
                unsigned uw = 0u;
                for (int t0 = 0; t0 < zn; t0 += kZBatch) {
                  float vv[kZBatch];
#pragma unroll
                  for (int u = 0; u < kZBatch; ++u) vv[u] = have && t0 + u < zn ? col[(size_t)(t0 + u) * P] : 0.0f;
                  unsigned ub = 0u;                      // fitted voxels of this batch
#pragma unroll
                  for (int u = 0; u < kZBatch; ++u) {
                    const int t = t0 + u;
                    if (t >= zn) break;
                    const int z = 32 * w + t;
                    if (have) {
                        const float v = vv[u] - R.sb_bias;
                        const float pv = P2 * fR[z];
                        const float ppv = (P2p * fRp[z]) * hp;
                        const bool clean = v >= 0.0f && !((nw >> t) & 1u);
                        if (!clean) lost += fR[z];
                        const bool use = clean && (pv > pthr || ppv > ppthr);
                        const float net = v - bpix;
                        if (STAGED) stage[(size_t)z * P + p] = use ? net : __int_as_float(0x7fc00000);
                        if (use) {
                            ub |= 1u << u;
                            a8[0] += (double)net;
                            a8[1] += (double)(pv + ppv);
                            a8[5] += (double)((pv * pv) * iv0);
                            a8[6] += (double)((pv * bref) * iv0);
                            a8[7] += 1.0;
                        }
                    }
                  }
                  uw |= ub << t0;
                  // warp-aggregated append of the batch's fitted voxels to the fit list: a lane's entries follow
                  // the entries of the lanes before it (one scan and one atomic per warp and batch)
                  const int c = __popc(ub);
                  int incl = c;
#pragma unroll
                  for (int o = 1; o < 32; o <<= 1) {
                      const int y = __shfl_up_sync(0xffffffffu, incl, o);
                      if (lane >= o) incl += y;
                  }
                  const int wtot = __shfl_sync(0xffffffffu, incl, 31);
                  if (wtot) {
                      int base = 0;
                      if (lane == 31) base = atomicAdd(&s_nlist, wtot);
                      base = __shfl_sync(0xffffffffu, base, 31);
                      int k = base + incl - c;
#pragma unroll
                      for (int u = 0; u < kZBatch; ++u) {
                          if (!((ub >> u) & 1u)) continue;
                          if (k < cap) {
                              ul_v[k] = (vv[u] - R.sb_bias) - bpix;
                              ul_i[k] = ((unsigned)(32 * w + t0 + u) << 16) | (unsigned)p;
                          }
                          ++k;
                      }
                  }
                }
                umw[w] = uw;
            }
            if (have) {
                const double tp = (double)P2 * r_all;
                a8[2] += tp;
                a8[3] += tp - (double)P2 * (double)lost;
                if (fg2) a8[4] += (double)P2 * r_fg;
                if (STAGED) {                    // the neighbour mask is not needed any more: keep the fit mask
                    nblo[p] = (unsigned long long)umw[0] | ((unsigned long long)umw[1] << 32);
                    if (nbhi) {                  // this pixel's bit only: other threads own the word's others
                        if (umw[2] & 1u) atomicOr(&nbhi[p >> 5], 1u << (p & 31));
                        else atomicAnd(&nbhi[p >> 5], ~(1u << (p & 31)));
                    }
                }
            }
        }
        block_sum<NT, 8>(a8, red, tot);
        if (threadIdx.x == 0) {
            const float I0 = (float)tot[0] / fmaxf((float)tot[1], 1e-6f);
            s_I = I0;
            s_Ip = I0 * hp;
        }
        __syncthreads();
    }
    const double s_net_use = tot[0];
    const float p_total = (float)tot[2], p_valid = (float)tot[3], p_fgn = (float)tot[4];
    const double a110 = fmax(tot[5], 1e-12), C0 = tot[6];
    const float nuse = (float)tot[7];
    const int nlist = s_nlist;
    const bool listed = nlist <= cap;

    // every fitted voxel of this thread: f(net, pv, ppv, bpix, bref)
    auto each_fitted = [&](auto&& f) {
        if (listed) {
            for (int k = threadIdx.x; k < nlist; k += NT) {
                const unsigned id = ul_i[k];
                const int z = (int)(id >> 16), p = (int)(id & 0xffffu);
                const float bref = brefs[p];
                f(ul_v[k], P2s[p] * fR[z], (P2ps[p] * fRp[z]) * hp, bg * bref, bref);
            }
            return;
        }
        for (int p = threadIdx.x; p < P; p += NT) {
            const float bref = brefs[p];
            const float bpix = bg * bref;
            const float P2 = P2s[p], P2p = P2ps[p];
            Mask65 nbm;
            nbm.lo = nblo[p];
            nbm.hi = hi_bit(p);
            for (int z = 0; z < Dz; ++z) {
                if (STAGED) {
                    if (!nbm.get(z)) continue;   // fit mask
                    f(stage[(size_t)z * P + p], P2 * fR[z], (P2p * fRp[z]) * hp, bpix, bref);
                    continue;
                }
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
                if (!(v >= 0.0f) || nbm.get(z)) continue;
                const float pv = P2 * fR[z];
                const float ppv = (P2p * fRp[z]) * hp;
                if (!(pv > pthr || ppv > ppthr)) continue;
                f(v - bpix, pv, ppv, bpix, bref);
            }
        }
    };

    // ---- IRLS: Poisson-weighted 2x2 normal equations, float64 sums, N_IRLS iterations; the last iteration's
    // weights also give C of the variance tail and the sum of the fitted profile values
    double a11 = 0.0, a12 = 0.0, a22 = 1.0, b1 = 0.0, b2 = 0.0, det2 = 1.0, Cc = 0.0, swp = 0.0;
    for (int it = 0; it < kIrls; ++it) {
        const bool last = it == kIrls - 1;
        const float I = s_I, Ip = s_Ip;
        const float Ipos = fmaxf(I, 0.0f), Ippos = fmaxf(Ip, 0.0f);
        double a7[7] = {0, 0, 0, 0, 0, 0, 0};   // a11, b1, a12, a22, b2, C, sum p
        each_fitted([&](float net, float pv, float ppv, float bpix, float bref) {
            float mu = bpix + Ipos * pv;
            if (has_p) mu = mu + Ippos * ppv;
            const float iv = __frcp_rn(gain * fmaxf(mu, kVarFloor));
            a7[0] += (double)((pv * pv) * iv);
            a7[1] += (double)((pv * net) * iv);
            if (has_p) {
                a7[2] += (double)((pv * ppv) * iv);
                a7[3] += (double)((ppv * ppv) * iv);
                a7[4] += (double)((ppv * net) * iv);
            }
            if (last) {
                a7[5] += (double)((pv * bref) * iv);
                a7[6] += (double)pv;
            }
        });
        block_sum<NT, 7>(a7, red, tot);
        a11 = tot[0];
        b1 = tot[1];
        if (has_p) {
            a12 = tot[2];
            a22 = tot[3];
            b2 = tot[4];
        } else {
            a12 = 0.0;
            a22 = 1.0;
            b2 = 0.0;
        }
        if (last) {
            Cc = tot[5];
            swp = tot[6];
        }
        det2 = fmax(a11 * a22 - a12 * a12, 1e-30);
        if (threadIdx.x == 0) {
            s_I = (float)((a22 * b1 - a12 * b2) / det2);
            s_Ip = (float)((a11 * b2 - a12 * b1) / det2 * (double)hp);
        }
        __syncthreads();
    }
    const float I = s_I, Ip = s_Ip;
    const float Ippos = fmaxf(Ip, 0.0f);
    const float pm = (float)swp / fmaxf(nuse, 1.0f);
    // mean residual over the fitted voxels (with a partner the residual removes the partner's fitted share)
    double s_resid = s_net_use;
    if (has_p) {
        double a1[1] = {0.0};
        each_fitted([&](float net, float pv, float ppv, float bpix, float bref) {
            a1[0] += (double)(net - Ippos * ppv);
        });
        block_sum<NT, 1>(a1, red, tot);
        s_resid = tot[0];
    }
    const float nm = (float)s_resid / fmaxf(nuse, 1.0f);
    // ---- profile / residual correlation ------------------------------------------------------------------------
    {
        double a3[3] = {0.0, 0.0, 0.0};
        each_fitted([&](float net, float pv, float ppv, float bpix, float bref) {
            const float resid = has_p ? net - Ippos * ppv : net;
            const float dp = pv - pm, dn = resid - nm;
            a3[0] += (double)(dp * dn);
            a3[1] += (double)(dp * dp);
            a3[2] += (double)(dn * dn);
        });
        block_sum<NT, 3>(a3, red, tot);
    }
    if (threadIdx.x == 0) {
        const double var_b = (double)gain * fmax((double)bg, (double)kVarFloor) / fmax((double)nbgv, 1.0);
        const double a11i = a22 / det2;
        const double varI = a11i + (Cc * a11i) * (Cc * a11i) * var_b;
        const double infl = a11i * a11;
        const double var0 = (1.0 / a110 + (C0 / a110) * (C0 / a110) * var_b) * fmax(infl, 1.0);
        const float sdd = (float)tot[0], spp = (float)tot[1], snn = (float)tot[2];
        O.iprf[row] = I;
        O.vprf[row] = (float)varI;
        O.vprf0[row] = (float)var0;
        O.corr[row] = sdd / sqrtf(fmaxf(spp * snn, 1e-20f));
        O.p_valid[row] = p_valid;
        O.p_total[row] = p_total;
        O.ipartner[row] = Ip;
        O.rho[row] = has_p ? (float)(a12 / sqrt(fmax(a11 * a22, 1e-30))) : 0.0f;
        O.p_fg[row] = p_fgn / fmaxf(p_total, 1e-9f);
    }
}

// Pass 2, one CTA per row of `order` (one shoebox shape group per launch).
template <int NT, bool STAGED>
__global__ void __launch_bounds__(NT, min_ctas<NT>()) k_pass2(XiDetector det_g, XiRows R, XiBlock B,
                                                              const float* __restrict__ arena,
                                                              const float* __restrict__ prof, XiPass2In I2,
                                                              XiPass2Out O, const int32_t* __restrict__ order,
                                                              int max_bx, int max_dz, int cap, int* status) {
    __shared__ __align__(8) unsigned long long s_bar;
    if (STAGED && threadIdx.x == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    unsigned phase = 0;
    pass2_row<NT, STAGED>(det_g, R, B, arena, prof, I2, O, order ? order[blockIdx.x] : blockIdx.x, max_bx, max_dz,
                          cap, status, &s_bar, phase);
}

// Pass 2 over a queue of (set, row) items (as k_pass1_q); a set's pass-1 outputs are its pass-2 inputs.
template <int NT, bool STAGED>
__global__ void __launch_bounds__(NT, min_ctas<NT>()) k_pass2_q(const XiRowSet* __restrict__ sets,
                                                                const int64_t* __restrict__ items, int n_items,
                                                                int max_bx, int max_dz, int max_k, int cap,
                                                                int* queue, int* status) {
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ XiRowSet s_set;
    __shared__ int s_item, s_cur;
    if (threadIdx.x == 0) {
        if (STAGED) mbar_init(&s_bar, 1);
        s_cur = -1;
    }
    unsigned phase = 0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) return;
        const int64_t v = items[it];
        const int set = (int)(v >> 32);
        if (set != s_cur) load_set(sets, set, &s_set, &s_cur);
        if (s_set.rows.K > max_k) {
            if (threadIdx.x == 0) atomicOr(status, 1);
            continue;
        }
        XiPass2In in;
        in.zeta = s_set.p1.zeta;
        in.seff = s_set.p1.seff;
        in.J = s_set.p1.J;
        in.u1 = s_set.p1.u1;
        in.u2 = s_set.p1.u2;
        in.bg = s_set.p1.bg;
        in.nbg = s_set.p1.nbg;
        pass2_row<NT, STAGED>(s_set.det, s_set.rows, s_set.blk, s_set.arena, s_set.prof, in, s_set.p2,
                              (int)(v & 0xffffffffll), max_bx, max_dz, cap, status, &s_bar, phase);
    }
}

// ==================================================================================================================
// gather and bin decode
// ==================================================================================================================
__device__ __forceinline__ float prepared_pixel(const XiFrames& F, const void* frame, int y, int x) {
    // one detector pixel of a frame as XPG's readers deliver it, with the mask ceiling applied
    if (y < 0 || y >= F.ny || x < 0 || x >= F.nx) return -1.0f;
    const size_t idx = (size_t)y * F.nx + x;
    float v;
    if (F.is_float) {
        v = ((const float*)frame)[idx];
    } else {
        const uint32_t r = ((const uint32_t*)frame)[idx];
        if (r == 0xFFFFFFFFu || r < F.min_valid) v = -1.0f;
        else if (r >= F.overload) v = -2.0f;
        else v = (float)r;
    }
    if (F.mask && F.mask[idx] == 0) v = fminf(v, -1.0f);
    return v;
}

// the raw value of a pixel known to be inside the frame, encoded as XPG's readers deliver it (mask applied later)
__device__ __forceinline__ float encode_raw(const XiFrames& F, uint32_t r) {
    if (r == 0xFFFFFFFFu || r < F.min_valid) return -1.0f;
    if (r >= F.overload) return -2.0f;
    return (float)r;
}

__device__ __forceinline__ float box_value(const XiFrames& F, const void* frame, int sy, int sx, int s) {
    if (s == 1) return prepared_pixel(F, frame, sy, sx);
    // s x s super-pixel (xpg/integrate.py:682-699): incomplete super-pixels at the far edges are masked
    if (sy < 0 || sx < 0 || sy >= F.ny / s || sx >= F.nx / s) return -1.0f;
    float sum = 0.0f, mn = 0.0f;
    for (int a = 0; a < s; ++a)
        for (int c = 0; c < s; ++c) {
            const float v = prepared_pixel(F, frame, sy * s + a, sx * s + c);
            if (a == 0 && c == 0) { sum = v; mn = v; }
            else { sum = sum + v; mn = fminf(mn, v); }
        }
    if (mn < 0.0f) return mn <= -1.5f ? -2.0f : -1.0f;
    return sum;
}

// The gather of one row's box from the frames of a wedge, by the whole CTA.
__device__ __forceinline__ void gather_row(const XiFrames& F, const XiGatherRows& G, float* __restrict__ arena,
                                           int32_t* __restrict__ cnt, int row) {
    const int iz0 = G.iz0[row], fb = G.fb[row], Dz = G.Dz[row], bx = G.bx[row];
    const int s = G.pxs ? G.pxs[row] : 1;
    const int ix0 = G.ix0[row], iy0 = G.iy0[row];
    const int P = bx * bx;
    const int span = Dz * fb;
    const int w0 = max(0, iz0 - F.first_fi), w1 = min(F.n_frames, iz0 + span - F.first_fi);
    float* dst = arena + G.sb_off[row];
    const size_t fstride = (size_t)F.ny * F.nx * (F.is_float ? sizeof(float) : sizeof(uint32_t));
    if (fb == 1 && s == 1) {
        // plain rows: a thread owns box pixels and reads a pixel's frames kGatherBatch at a time (independent loads
        // in flight); the pixel's bounds and mask are looked up once
        const size_t fpix = (size_t)F.ny * F.nx;
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            const int y = iy0 + p / bx, x = ix0 + p % bx;
            const bool inside = y >= 0 && y < F.ny && x >= 0 && x < F.nx;
            const size_t idx = inside ? (size_t)y * F.nx + x : 0;
            const bool masked = inside && F.mask && F.mask[idx] == 0;
            const int k0 = F.first_fi - iz0;                  // box frame of wedge frame 0
            for (int w = w0; w < w1; w += kGatherBatch) {
                float vv[kGatherBatch];
#pragma unroll
                for (int u = 0; u < kGatherBatch; ++u) {
                    vv[u] = -1.0f;
                    const int ww = w + u;
                    if (inside && ww < w1) {
                        const size_t o = (size_t)ww * fpix + idx;
                        vv[u] = F.is_float ? ((const float*)F.data)[o] : encode_raw(F, ((const uint32_t*)F.data)[o]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kGatherBatch; ++u) {
                    const int ww = w + u;
                    if (ww >= w1 || (F.frame_ok && !F.frame_ok[ww])) continue;
                    const float v = masked ? fminf(vv[u], -1.0f) : vv[u];
                    dst[(size_t)(k0 + ww) * P + p] = v + kSbOff;
                }
            }
        }
        return;
    }
    for (int w = w0; w < w1; ++w) {
        if (F.frame_ok && !F.frame_ok[w]) continue;
        const int fi = F.first_fi + w;
        const int k = fi - iz0;
        const void* frame = (const char*)F.data + (size_t)w * fstride;
        if (fb == 1) {
            float* slot = dst + (size_t)k * P;
            for (int p = threadIdx.x; p < P; p += blockDim.x) {
                const int i = p % bx, j = p / bx;
                slot[p] = box_value(F, frame, iy0 + j, ix0 + i, s) + kSbOff;
            }
        } else {
            const int kb = k / fb;
            float* slot = dst + (size_t)kb * P;
            for (int p = threadIdx.x; p < P; p += blockDim.x) {
                const int i = p % bx, j = p / bx;
                float v = box_value(F, frame, iy0 + j, ix0 + i, s);
                if (v < 0.0f) v = (v == -2.0f) ? __int_as_float(0x7fc00000) : __int_as_float(0x7f800000);
                slot[p] = slot[p] + v;
            }
            if (threadIdx.x == 0) cnt[G.cnt_off[row] + kb] += 1;
        }
    }
}

__global__ void k_gather(XiFrames F, XiGatherRows G, float* __restrict__ arena, int32_t* __restrict__ cnt,
                         const int32_t* __restrict__ order) {
    gather_row(F, G, arena, cnt, order ? order[blockIdx.x] : blockIdx.x);
}

// The gather of one wedge with the frames and rows read from a device descriptor when the kernel runs, so that one
// launch captured in a CUDA graph serves every wedge of a block: CTAs stride over the step's rows.
__global__ void k_gather_step(const XiGatherStep* __restrict__ step, XiGatherRows G, float* __restrict__ arena,
                              int32_t* __restrict__ cnt) {
    const XiFrames F = step->frames;
    const int n = step->n_order;
    if (F.n_frames <= 0) return;
    for (int k = blockIdx.x; k < n; k += gridDim.x) gather_row(F, G, arena, cnt, step->order[k]);
}


__global__ void k_decode_bins(XiGatherRows G, float* __restrict__ arena, const int32_t* __restrict__ cnt) {
    const int row = G.order ? G.order[blockIdx.x] : blockIdx.x;
    if (G.cnt_off[row] < 0) return;
    const int Dz = G.Dz[row], bx = G.bx[row], fb = G.fb[row];
    const int P = bx * bx;
    float* a = arena + G.sb_off[row];
    const int32_t* c = cnt + G.cnt_off[row];
    for (int v = threadIdx.x; v < Dz * P; v += blockDim.x) {
        const int z = v / P;
        float x = a[v];
        if (isnan(x)) x = -2.0f;
        else if (isinf(x)) x = -1.0f;
        x = x + kSbOff;
        if (c[z] < fb) x = 0.0f;
        a[v] = x;
    }
}

// zero the arena slots of the listed rows (rows the gather does not write in full: binned rows accumulate, rows whose
// frames reach beyond the run's). A row's slot is Dz * bx^2 floats rounded up to 4 and starts on 16 bytes.
__global__ void k_zero_rows(XiGatherRows G, float* __restrict__ arena) {
    const int row = G.order ? G.order[blockIdx.x] : blockIdx.x;
    const int64_t v = (int64_t)G.Dz[row] * G.bx[row] * G.bx[row];
    const int64_t n4 = (v + 3) / 4;
    float4* a = reinterpret_cast<float4*>(arena + G.sb_off[row]);
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int64_t i = threadIdx.x; i < n4; i += blockDim.x) a[i] = z;
}

// ==================================================================================================================
// profile accumulation and finalisation
// ==================================================================================================================
__global__ void k_accumulate(XiRows R, XiPass1Out O, const uint8_t* __restrict__ sel, int strong_test,
                             int n_regions, double* __restrict__ num, double* __restrict__ den) {
    const int row = R.order ? R.order[blockIdx.x] : blockIdx.x;
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        bool ok = true;
        if (strong_test) {
            // strong, fully recorded, unobstructed (xpg/integrate.py:531-533), float64 on the float32 outputs
            const double isum = (double)O.isum[row], vs = (double)O.vsum[row];
            ok = (isum > 0.0) && (isum / sqrt(fmax(vs, 1e-6)) > 10.0) && O.n_over[row] == 0 &&
                 (double)O.frac_rec[row] > 0.95 && O.n_fg_nb[row] == 0 && O.n_fg_masked[row] == 0;
        }
        if (sel && !sel[row]) ok = false;
        const int reg = R.region[row];
        if (reg < 0 || reg >= n_regions) ok = false;
        s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return;
    const int bx = R.bx[row];
    const int P = bx * bx;
    const int64_t po = R.pix_off[row];
    const float isum = fmaxf(O.isum[row], 1e-6f);
    const float seff = O.seff[row];
    const float s2 = seff * seff;
    double* nr = num + (size_t)R.region[row] * XI_GRID * XI_GRID;
    double* dr = den + (size_t)R.region[row] * XI_GRID * XI_GRID;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const float dens = (O.img2[po + p] / isum) / fmaxf(O.J[po + p] / s2, 1e-12f);
        GridCell g = grid_cell(O.u1[po + p], O.u2[po + p]);
        if (!(O.all_valid2[po + p] && g.inside)) continue;
        const float w00 = (1.0f - g.t1) * (1.0f - g.t2), w10 = g.t1 * (1.0f - g.t2);
        const float w01 = (1.0f - g.t1) * g.t2, w11 = g.t1 * g.t2;
        const int b = g.i2 * XI_GRID + g.i1;
        atomicAdd(nr + b, (double)(w00 * dens));
        atomicAdd(dr + b, (double)w00);
        atomicAdd(nr + b + 1, (double)(w10 * dens));
        atomicAdd(dr + b + 1, (double)w10);
        atomicAdd(nr + b + XI_GRID, (double)(w01 * dens));
        atomicAdd(dr + b + XI_GRID, (double)w01);
        atomicAdd(nr + b + XI_GRID + 1, (double)(w11 * dens));
        atomicAdd(dr + b + XI_GRID + 1, (double)w11);
    }
}

__global__ void k_finalize(const double* __restrict__ num, const double* __restrict__ den, float* __restrict__ prof) {
    // one CTA per region (xpg/integrate.py:546-555); the Gaussian prior is float32-rounded as XPG's table
    const int r = blockIdx.x;
    constexpr int G2 = XI_GRID * XI_GRID;
    __shared__ double pr[G2];
    __shared__ double part[32];
    const double du = (9.0 / (XI_GRID - 1)) * (9.0 / (XI_GRID - 1));
    for (int q = threadIdx.x; q < G2; q += blockDim.x) {
        const int iy = q / XI_GRID, ix = q % XI_GRID;
        // numpy.linspace(-4.5, 4.5, 41): i * step + start, the last point exactly 4.5
        const double step = 9.0 / (XI_GRID - 1);
        const double u1 = ix == XI_GRID - 1 ? 4.5 : (double)ix * step + (-4.5);
        const double u2 = iy == XI_GRID - 1 ? 4.5 : (double)iy * step + (-4.5);
        const float gauss = (float)(exp(-0.5 * (u1 * u1 + u2 * u2)) / (2.0 * 3.141592653589793));
        const float g3 = 3.0f * gauss;                 // XPG: 3.0 * (float32 table) stays float32
        const double n = num[(size_t)r * G2 + q], d = den[(size_t)r * G2 + q];
        const double dens = d > 0.0 ? n / fmax(d, 1e-12) : 0.0;
        const double emp = fmax(dens, 0.0);
        const double v = (d * emp + (double)g3) / (d + 3.0);
        pr[q] = v;
    }
    __syncthreads();
    // sum in index order by one warp (fixed order), then normalise
    if (threadIdx.x < 32) {
        double s = 0.0;
        for (int q = threadIdx.x; q < G2; q += 32) s += pr[q];
        part[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < 32; ++q) s += part[q];
        part[0] = fmax(s * du, 1e-12);
    }
    __syncthreads();
    const double norm = part[0];
    for (int q = threadIdx.x; q < G2; q += blockDim.x) prof[(size_t)r * G2 + q] = (float)(pr[q] / norm);
}

// status word of the kernels (rows skipped for an unsupported shape)
__device__ int g_status = 0;

int* status_ptr() {
    static int* p = nullptr;
    int dev = -1;
    cudaGetDevice(&dev);
    static int pdev = -2;
    if (p == nullptr || pdev != dev) {
        if (cudaGetSymbolAddress((void**)&p, g_status) != cudaSuccess) return nullptr;
        pdev = dev;
    }
    return p;
}

int rows_check(const XiRows* R) {
    if (!R) return fail(XI_E_ARG, "rows: null");
    if (R->n < 0 || (R->order && R->n_order < 0)) return fail(XI_E_ARG, "rows: negative count");
    if (R->K < 0 || R->K > XI_MAX_K) return fail(XI_E_LIMIT, "rows: neighbour columns beyond XI_MAX_K");
    if (R->max_bx < 3 || R->max_bx > XI_MAX_BX || R->max_dz < 1 || R->max_dz > XI_MAX_DZ)
        return fail(XI_E_LIMIT, "rows: max_bx / max_dz outside 3..97 / 1..65");
    return XI_OK;
}

template <int NT, bool STAGED>
int launch_pass1(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena, XiPass1Out* O,
                 cudaStream_t s, int nblk) {
    const size_t P = (size_t)R->max_bx * R->max_bx;
    size_t sm = pass1_pix_bytes((int)P) + (STAGED ? (P * R->max_dz * sizeof(float) + 15) / 16 * 16 : 0) +
                nb_bytes(R->K, R->max_bx, R->max_dz);
    cudaFuncSetAttribute(k_pass1<NT, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k_pass1<NT, STAGED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    k_pass1<NT, STAGED><<<nblk, NT, sm, s>>>(*det, *R, *B, arena, *O, R->order, R->max_bx, R->max_dz,
                                              status_ptr());
    return cuda_check("xi_pass1");
}

template <int NT, bool STAGED>
int launch_pass2(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena, const float* prof,
                 const XiPass2In* in, XiPass2Out* O, cudaStream_t s, int nblk, int cap) {
    const size_t P = (size_t)R->max_bx * R->max_bx;
    size_t sm = pass2_stage_offset((int)P, R->max_dz, cap) + (STAGED ? (P * R->max_dz * sizeof(float) + 15) / 16 * 16 : 0) +
                nb_bytes(R->K, R->max_bx, R->max_dz);
    cudaFuncSetAttribute(k_pass2<NT, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k_pass2<NT, STAGED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    k_pass2<NT, STAGED><<<nblk, NT, sm, s>>>(*det, *R, *B, arena, prof, *in, *O, R->order, R->max_bx, R->max_dz,
                                              cap, status_ptr());
    return cuda_check("xi_pass2");
}

__global__ void k_zero_int(int* p) { *p = 0; }

// Resident CTAs of a persistent launch: as many as the SMs hold at once (at least one).
template <typename K>
int resident_grid(K kernel, int nt, size_t smem, int n_items) {
    int dev = 0, n_sm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nt, smem) != cudaSuccess)
        return -1;
    const long long g = (long long)(per_sm > 0 ? per_sm : 1) * n_sm;
    return (int)(g < n_items ? g : n_items);
}

template <int NT, bool STAGED>
int launch_pass1_q(const XiRowSet* sets, const int64_t* items, int n_items, int max_bx, int max_dz, int K, int* queue,
                   cudaStream_t s) {
    const size_t P = (size_t)max_bx * max_bx;
    const size_t sm = pass1_pix_bytes((int)P) + (STAGED ? (P * max_dz * sizeof(float) + 15) / 16 * 16 : 0) +
                      nb_bytes(K, max_bx, max_dz);
    cudaFuncSetAttribute(k_pass1_q<NT, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k_pass1_q<NT, STAGED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    const int grid = resident_grid(k_pass1_q<NT, STAGED>, NT, sm, n_items);
    if (grid <= 0) return cuda_check("xi_pass1_batched: occupancy");
    k_zero_int<<<1, 1, 0, s>>>(queue);
    k_pass1_q<NT, STAGED><<<grid, NT, sm, s>>>(sets, items, n_items, max_bx, max_dz, K, queue, status_ptr());
    return cuda_check("xi_pass1_batched");
}

template <int NT, bool STAGED>
int launch_pass2_q(const XiRowSet* sets, const int64_t* items, int n_items, int max_bx, int max_dz, int K, int cap,
                   int* queue, cudaStream_t s) {
    const size_t P = (size_t)max_bx * max_bx;
    const size_t sm = pass2_stage_offset((int)P, max_dz, cap) +
                      (STAGED ? (P * max_dz * sizeof(float) + 15) / 16 * 16 : 0) + nb_bytes(K, max_bx, max_dz);
    cudaFuncSetAttribute(k_pass2_q<NT, STAGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaFuncSetAttribute(k_pass2_q<NT, STAGED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    const int grid = resident_grid(k_pass2_q<NT, STAGED>, NT, sm, n_items);
    if (grid <= 0) return cuda_check("xi_pass2_batched: occupancy");
    k_zero_int<<<1, 1, 0, s>>>(queue);
    k_pass2_q<NT, STAGED><<<grid, NT, sm, s>>>(sets, items, n_items, max_bx, max_dz, K, cap, queue, status_ptr());
    return cuda_check("xi_pass2_batched");
}

// Dynamic shared memory available beside the kernels' static arrays (bytes).
constexpr size_t kStageBudget = 190 * 1024;

// Launch tuning (xi_tune): the largest shoebox each pass stages in shared memory, and the fit-list capacity of
// pass 2. Larger staging overlaps the box read with the set-up but costs resident CTAs per SM.
size_t g_stage_max[2] = {48 * 1024, 48 * 1024};
int g_list_cap[2] = {2048, 8192};   // boxes up to XI_PASS2_LARGE_VOXELS voxels, larger boxes
int g_wide_nt = 256;          // threads per CTA of the pass kernels for boxes over 200 pixels (128 or 256)

// Pass 1 stages boxes of up to g_stage_max[0] bytes when they fit beside the per-pixel tables.
bool pass1_staged(size_t P, int max_dz) {
    return P * max_dz * sizeof(float) <= g_stage_max[0] &&
           pass1_pix_bytes((int)P) + P * max_dz * sizeof(float) + 16 <= kStageBudget;
}

// Pass 2's shared-memory plan for boxes up to max_bx pixels a side and max_dz bins with K neighbour columns: whether the box is
// staged, and the fit list's capacity. The largest boxes (up to 97 px, 65 frames) take what the device allows a CTA
// beyond the kernel's static arrays and the neighbour tables, not the default budget. The fit list holds up to every
// voxel of small boxes and g_list_cap fitted voxels of large ones (the second capacity for launches whose largest box
// exceeds XI_PASS2_LARGE_VOXELS voxels or XI_PASS2_LARGE_DEPTH bins: such boxes fit more voxels (a deep rocking curve
// keeps many frames above the profile threshold), whose rows would otherwise overflow a short list and
// fit from the box in each later pass; fewer CTAs per SM pay less there; less when shared memory is short; rows whose list
// overflows fit from the box); the box is staged only when small (it is read once: staging buys the copy's overlap
// with the set-up, not re-reads).
int pass2_plan(int max_bx, int max_dz, int K, const char* who, bool* staged, int* cap_out) {
    const size_t P = (size_t)max_bx * max_bx;
    const size_t V = P * max_dz;
    size_t budget = kStageBudget;
    if (pass2_pix_bytes((int)P, max_dz) + pass2_list_bytes(0) > budget) {
        int dev = 0, optin = 0;
        cudaFuncAttributes fa, fq;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
            cudaFuncGetAttributes(&fa, k_pass2<256, false>) != cudaSuccess ||
            cudaFuncGetAttributes(&fq, k_pass2_q<256, false>) != cudaSuccess)
            return cuda_check(who);
        const size_t st = fa.sharedSizeBytes > fq.sharedSizeBytes ? fa.sharedSizeBytes : fq.sharedSizeBytes;
        const size_t fixed = st + nb_bytes(K, max_bx, max_dz);
        budget = (size_t)optin > fixed ? (size_t)optin - fixed : 0;
        if (pass2_pix_bytes((int)P, max_dz) + pass2_list_bytes(0) > budget)
            return fail(XI_E_LIMIT, "pass 2: box too large (per-pixel tables exceed shared memory)");
    }
    const size_t fit = (budget - pass2_pix_bytes((int)P, max_dz)) / 8 / 4 * 4;
    const bool large = V > (size_t)XI_PASS2_LARGE_VOXELS || max_dz > XI_PASS2_LARGE_DEPTH;
    const size_t want = (size_t)g_list_cap[large ? 1 : 0];
    size_t capz = V < want ? V : want;
    if (capz > fit) capz = fit;
    *cap_out = (int)capz;
    const size_t base = pass2_stage_offset((int)P, max_dz, *cap_out);
    if (base > budget) return fail(XI_E_LIMIT, "pass 2: shared memory");
    *staged = V * sizeof(float) <= g_stage_max[1] && base + V * sizeof(float) + 16 <= budget;
    return XI_OK;
}

}  // namespace

// ==================================================================================================================
// C ABI
// ==================================================================================================================
extern "C" {

const char* xi_last_error(void) { return g_err; }

int xi_version(void) { return 3; }

int xi_tune(int key, long long value) {
    if (key == XI_TUNE_PASS1_STAGE_BYTES || key == XI_TUNE_PASS2_STAGE_BYTES) {
        if (value < 0 || value > (long long)kStageBudget) return fail(XI_E_LIMIT, "xi_tune: staging bytes");
        g_stage_max[key == XI_TUNE_PASS1_STAGE_BYTES ? 0 : 1] = (size_t)value;
        return XI_OK;
    }
    if (key == XI_TUNE_WIDE_THREADS) {
        if (value != 128 && value != 256) return fail(XI_E_LIMIT, "xi_tune: threads per CTA (128 or 256)");
        g_wide_nt = (int)value;
        return XI_OK;
    }
    if (key == XI_TUNE_PASS2_LIST_CAP || key == XI_TUNE_PASS2_LIST_CAP_LARGE) {
        if (value < 0 || value > 16384) return fail(XI_E_LIMIT, "xi_tune: list capacity");
        g_list_cap[key == XI_TUNE_PASS2_LIST_CAP ? 0 : 1] = (int)value;
        return XI_OK;
    }
    return fail(XI_E_ARG, "xi_tune: unknown key");
}

int xi_status(void* stream) {
    int* p = status_ptr();
    if (!p) return fail(XI_E_CUDA, "status word unavailable");
    int h = 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(&h, p, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return cuda_check("xi_status");
    if (h) {
        int zero = 0;
        cudaMemcpyAsync(p, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
        cudaStreamSynchronize(s);
        return fail(XI_E_SHAPE, "a row's shoebox shape exceeded the call's shape hint; the row was skipped");
    }
    return XI_OK;
}


int xi_status_copy(int* host_dst, void* stream) {
    int* p = status_ptr();
    if (!p) return fail(XI_E_CUDA, "status word unavailable");
    if (!host_dst) return fail(XI_E_ARG, "xi_status_copy: null destination");
    if (cudaMemcpyAsync(host_dst, p, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess)
        return cuda_check("xi_status_copy");
    return XI_OK;
}


int xi_pass1(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena, XiPass1Out* O,
             void* stream) {
    if (!det || !B || !arena || !O) return fail(XI_E_ARG, "xi_pass1: null argument");
    int rc = rows_check(R);
    if (rc) return rc;
    const int nblk = R->order ? R->n_order : R->n;
    if (nblk == 0) return XI_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t P = (size_t)R->max_bx * R->max_bx;
    const bool staged = pass1_staged(P, R->max_dz);
    if (staged) {
        if (P <= 96) return launch_pass1<64, true>(det, R, B, arena, O, s, nblk);
        if (P <= 200 || g_wide_nt == 128) return launch_pass1<128, true>(det, R, B, arena, O, s, nblk);
        return launch_pass1<256, true>(det, R, B, arena, O, s, nblk);
    }
    if (P <= 96) return launch_pass1<64, false>(det, R, B, arena, O, s, nblk);
    if (P <= 200 || g_wide_nt == 128) return launch_pass1<128, false>(det, R, B, arena, O, s, nblk);
    return launch_pass1<256, false>(det, R, B, arena, O, s, nblk);
}


int xi_pass2(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena, const float* prof,
             const XiPass2In* in, XiPass2Out* O, void* stream) {
    if (!det || !B || !arena || !prof || !in || !O) return fail(XI_E_ARG, "xi_pass2: null argument");
    int rc = rows_check(R);
    if (rc) return rc;
    const int nblk = R->order ? R->n_order : R->n;
    if (nblk == 0) return XI_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t P = (size_t)R->max_bx * R->max_bx;
    bool staged = false;
    int cap = 0;
    rc = pass2_plan(R->max_bx, R->max_dz, R->K, "xi_pass2", &staged, &cap);
    if (rc) return rc;
    if (staged) {
        if (P <= 96) return launch_pass2<64, true>(det, R, B, arena, prof, in, O, s, nblk, cap);
        if (P <= 200 || g_wide_nt == 128) return launch_pass2<128, true>(det, R, B, arena, prof, in, O, s, nblk, cap);
        return launch_pass2<256, true>(det, R, B, arena, prof, in, O, s, nblk, cap);
    }
    if (P <= 96) return launch_pass2<64, false>(det, R, B, arena, prof, in, O, s, nblk, cap);
    if (P <= 200 || g_wide_nt == 128) return launch_pass2<128, false>(det, R, B, arena, prof, in, O, s, nblk, cap);
    return launch_pass2<256, false>(det, R, B, arena, prof, in, O, s, nblk, cap);
}

static int batched_check(const XiRowSet* sets, const int64_t* items, int n_items, int max_bx, int max_dz, int max_k,
                         int* queue, const char* who) {
    if (n_items < 0) return fail(XI_E_ARG, who);
    if (n_items && (!sets || !items || !queue)) return fail(XI_E_ARG, who);
    if (max_bx < 3 || max_bx > XI_MAX_BX || max_dz < 1 || max_dz > XI_MAX_DZ || max_k < 0 || max_k > XI_MAX_K)
        return fail(XI_E_LIMIT, "batched pass: max_bx / max_dz / max_k outside 3..97 / 1..65 / 0..16");
    return XI_OK;
}

int xi_pass1_batched(const XiRowSet* sets, const int64_t* items, int n_items, int max_bx, int max_dz, int max_k,
                     int* queue, void* stream) {
    int rc = batched_check(sets, items, n_items, max_bx, max_dz, max_k, queue, "xi_pass1_batched: bad argument");
    if (rc || n_items == 0) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t P = (size_t)max_bx * max_bx;
    if (pass1_staged(P, max_dz)) {
        if (P <= 96) return launch_pass1_q<64, true>(sets, items, n_items, max_bx, max_dz, max_k, queue, s);
        if (P <= 200 || g_wide_nt == 128) return launch_pass1_q<128, true>(sets, items, n_items, max_bx, max_dz, max_k, queue, s);
        return launch_pass1_q<256, true>(sets, items, n_items, max_bx, max_dz, max_k, queue, s);
    }
    if (P <= 96) return launch_pass1_q<64, false>(sets, items, n_items, max_bx, max_dz, max_k, queue, s);
    if (P <= 200 || g_wide_nt == 128) return launch_pass1_q<128, false>(sets, items, n_items, max_bx, max_dz, max_k, queue, s);
    return launch_pass1_q<256, false>(sets, items, n_items, max_bx, max_dz, max_k, queue, s);
}

int xi_pass2_batched(const XiRowSet* sets, const int64_t* items, int n_items, int max_bx, int max_dz, int max_k,
                     int* queue, void* stream) {
    int rc = batched_check(sets, items, n_items, max_bx, max_dz, max_k, queue, "xi_pass2_batched: bad argument");
    if (rc || n_items == 0) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t P = (size_t)max_bx * max_bx;
    bool staged = false;
    int cap = 0;
    rc = pass2_plan(max_bx, max_dz, max_k, "xi_pass2_batched", &staged, &cap);
    if (rc) return rc;
    if (staged) {
        if (P <= 96) return launch_pass2_q<64, true>(sets, items, n_items, max_bx, max_dz, max_k, cap, queue, s);
        if (P <= 200 || g_wide_nt == 128) return launch_pass2_q<128, true>(sets, items, n_items, max_bx, max_dz, max_k, cap, queue, s);
        return launch_pass2_q<256, true>(sets, items, n_items, max_bx, max_dz, max_k, cap, queue, s);
    }
    if (P <= 96) return launch_pass2_q<64, false>(sets, items, n_items, max_bx, max_dz, max_k, cap, queue, s);
    if (P <= 200 || g_wide_nt == 128) return launch_pass2_q<128, false>(sets, items, n_items, max_bx, max_dz, max_k, cap, queue, s);
    return launch_pass2_q<256, false>(sets, items, n_items, max_bx, max_dz, max_k, cap, queue, s);
}

int xi_gather(const XiFrames* F, const XiGatherRows* G, float* arena, int32_t* cnt, void* stream) {
    if (!F || !G || !arena || !F->data) return fail(XI_E_ARG, "xi_gather: null argument");
    if (F->n_frames < 0 || F->ny <= 0 || F->nx <= 0 || G->n < 0) return fail(XI_E_ARG, "xi_gather: bad sizes");
    const int nblk = G->order ? G->n_order : G->n;
    if (nblk == 0 || F->n_frames == 0) return XI_OK;
    k_gather<<<nblk, 128, 0, (cudaStream_t)stream>>>(*F, *G, arena, cnt, G->order);
    return cuda_check("xi_gather");
}

int xi_gather_step(const XiGatherStep* step, const XiGatherRows* G, float* arena, int32_t* cnt, int grid,
                   void* stream) {
    if (!step || !G || !arena) return fail(XI_E_ARG, "xi_gather_step: null argument");
    if (grid <= 0 || G->n < 0) return fail(XI_E_ARG, "xi_gather_step: bad sizes");
    k_gather_step<<<grid, 128, 0, (cudaStream_t)stream>>>(step, *G, arena, cnt);
    return cuda_check("xi_gather_step");
}

int xi_decode_bins(const XiGatherRows* G, float* arena, const int32_t* cnt, void* stream) {
    if (!G || !arena || !cnt) return fail(XI_E_ARG, "xi_decode_bins: null argument");
    if (G->n == 0) return XI_OK;
    const int nblk = G->order ? G->n_order : G->n;
    if (nblk <= 0) return XI_OK;
    k_decode_bins<<<nblk, 256, 0, (cudaStream_t)stream>>>(*G, arena, cnt);
    return cuda_check("xi_decode_bins");
}

int xi_zero_rows(const XiGatherRows* G, float* arena, void* stream) {
    if (!G || !arena) return fail(XI_E_ARG, "xi_zero_rows: null argument");
    const int nblk = G->order ? G->n_order : G->n;
    if (nblk <= 0) return XI_OK;
    if (((uintptr_t)arena & 15) != 0) return fail(XI_E_ARG, "xi_zero_rows: arena not on 16 bytes");
    k_zero_rows<<<nblk, 256, 0, (cudaStream_t)stream>>>(*G, arena);
    return cuda_check("xi_zero_rows");
}

int xi_accumulate(const XiRows* R, const XiPass1Out* p1, const uint8_t* sel, int strong_test, int n_regions,
                  double* num, double* den, void* stream) {
    if (!R || !p1 || !num || !den) return fail(XI_E_ARG, "xi_accumulate: null argument");
    if (n_regions <= 0) return fail(XI_E_ARG, "xi_accumulate: n_regions");
    const int nblk = R->order ? R->n_order : R->n;
    if (nblk == 0) return XI_OK;
    k_accumulate<<<nblk, 128, 0, (cudaStream_t)stream>>>(*R, *p1, sel, strong_test, n_regions, num, den);
    return cuda_check("xi_accumulate");
}

int xi_finalize_profiles(const double* num, const double* den, int n_regions, float* prof, void* stream) {
    if (!num || !den || !prof || n_regions <= 0) return fail(XI_E_ARG, "xi_finalize_profiles: bad argument");
    k_finalize<<<n_regions, 256, 0, (cudaStream_t)stream>>>(num, den, prof);
    return cuda_check("xi_finalize_profiles");
}

}  // extern "C"

int xi_fail(int code, const char* msg) { return fail(code, msg); }
int xi_cuda_check(const char* where) { return cuda_check(where); }
