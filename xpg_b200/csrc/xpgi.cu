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
    float dx2[XI_MAX_K][XI_MAX_BX];
    float dy2[XI_MAX_K][XI_MAX_BX];
    float dz2[XI_MAX_K][XI_MAX_DZ];
};

// Neighbour columns whose ellipsoid reaches the box (the separable pre-test of xpg/integrate_kernels.py:192-203;
// skipping the others is exact) and their per-axis terms.
__device__ void neighbour_setup(const XiRows& R, int row, int Dz, int bx, const float* xs, const float* ys,
                                const float* zzs, bool skip_first, NbShared& nb) {
    const int K = R.K;
    if (threadIdx.x == 0) {
        int n = 0;
        for (int k = 0; k < K; ++k) {
            if (k == 0 && skip_first) continue;
            float nx_ = R.nbx[(size_t)row * K + k], ny_ = R.nby[(size_t)row * K + k];
            float nz_ = R.nbz[(size_t)row * K + k];
            float sx = R.nbsx[(size_t)row * K + k], sz = R.nbsz[(size_t)row * K + k];
            float mx = (fminf(fmaxf(nx_, xs[0]), xs[bx - 1]) - nx_) / sx;
            float my = (fminf(fmaxf(ny_, ys[0]), ys[bx - 1]) - ny_) / sx;
            float mz = (fminf(fmaxf(nz_, zzs[0]), zzs[Dz - 1]) - nz_) / sz;
            if ((mx * mx + my * my) + mz * mz < 1.0f) nb.act[n++] = k;
        }
        nb.nact = n;
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
            nb.dx2[a][i] = dx * dx;
            nb.dy2[a][i] = dy * dy;
        }
        for (int z = threadIdx.x; z < Dz; z += blockDim.x) {
            float dz = (zzs[z] - nz_) / sz;
            nb.dz2[a][z] = dz * dz;
        }
    }
    __syncthreads();
}

// frames of pixel (i, j) inside any active neighbour's ellipsoid: ((dx^2 + dy^2) + dz^2 < 1)
__device__ __forceinline__ Mask65 neighbour_frames(const NbShared& nb, int i, int j, int Dz) {
    Mask65 m;
    m.clear();
    for (int a = 0; a < nb.nact; ++a) {
        float dxy = nb.dx2[a][i] + nb.dy2[a][j];
        for (int z = 0; z < Dz; ++z)
            if (dxy + nb.dz2[a][z] < 1.0f) m.set(z);
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
// pass 1
// ==================================================================================================================
template <int NT>
__global__ void __launch_bounds__(NT) k_pass1(XiDetector det, XiRows R, XiBlock B, const float* __restrict__ arena,
                                              XiPass1Out O, const int32_t* __restrict__ order, int max_bx,
                                              int max_dz, int* status) {
    extern __shared__ float dyn[];
    __shared__ float xs[XI_MAX_BX], ys[XI_MAX_BX];
    __shared__ float fR[XI_MAX_DZ], fzz[XI_MAX_DZ], fe3[XI_MAX_DZ];
    __shared__ NbShared nb;
    __shared__ float s_e1[3], s_e2[3], s_S[3], s_zeta, s_seff, s_b;
    __shared__ unsigned long long s_fgz_lo, s_rec_lo;
    __shared__ unsigned s_fgz_hi, s_rec_hi;
    __shared__ double red[NT / 32 * 16];
    __shared__ double tot[16];
    __shared__ float fzw[NT / 32][XI_MAX_DZ];

    const int row = order ? order[blockIdx.x] : blockIdx.x;
    const int Dz = R.Dz[row], bx = R.bx[row];
    if (Dz < 1 || Dz > max_dz || bx < 3 || bx > max_bx) {
        if (threadIdx.x == 0) atomicOr(status, 1);
        return;
    }
    const int P = bx * bx;
    float* u1s = dyn;
    float* u2s = dyn + P;
    const int pxs = R.pxs ? R.pxs[row] : 1;
    const int ix0 = R.ix0[row], iy0 = R.iy0[row], iz0 = R.iz0[row];
    const float fb = R.fb[row];
    const float phi = R.phi[row];
    const float* sb = arena + R.sb_off[row];
    const int64_t po = R.pix_off[row], fo = R.frm_off[row];
    const float gain = B.gain;

    if (threadIdx.x == 0) {
        float S[3] = {R.S[3 * row], R.S[3 * row + 1], R.S[3 * row + 2]};
        float e1[3], e2[3], zeta;
        kabsch_frame(S, B.s0, B.axis, e1, e2, &zeta);
        for (int c = 0; c < 3; ++c) { s_e1[c] = e1[c]; s_e2[c] = e2[c]; s_S[c] = S[c]; }
        s_zeta = zeta;
        s_fgz_lo = 0ull; s_fgz_hi = 0u; s_rec_lo = 0ull; s_rec_hi = 0u;
    }
    for (int i = threadIdx.x; i < bx; i += NT) {
        xs[i] = box_coord(ix0, i, pxs);
        ys[i] = box_coord(iy0, i, pxs);
    }
    for (int z = threadIdx.x; z < Dz; z += NT) fzz[z] = (float)iz0 + fb * ((float)z + 0.5f);
    __syncthreads();
    const float zeta = s_zeta;
    // frame terms: rocking-curve fractions, e3 of the bin centres
    for (int z = threadIdx.x; z < Dz; z += NT) {
        float lo, hi;
        bin_limits(iz0, fb, z, B.frames_phi0, B.osc, &lo, &hi);
        fR[z] = rocking_fraction(lo, hi, phi, zeta, B.sm, B.rcw);
        float phic = 0.5f * (lo + hi);
        fe3[z] = zeta * (phic - phi);
    }
    {
        float e1[3] = {s_e1[0], s_e1[1], s_e1[2]}, e2[3] = {s_e2[0], s_e2[1], s_e2[2]};
        float S[3] = {s_S[0], s_S[1], s_S[2]};
        box_geometry(det, S, e1, e2, bx, xs, ys, B.sd, u1s, u2s, O.J + po, nullptr, &s_seff);
    }
    // foreground frames: R >= 1e-3 * Rmax + 1e-6
    if (threadIdx.x == 0) {
        float Rmax = fR[0];
        for (int z = 1; z < Dz; ++z) Rmax = fmaxf(Rmax, fR[z]);
        float thr = 1e-3f * Rmax + 1e-6f;
        Mask65 m;
        m.clear();
        for (int z = 0; z < Dz; ++z)
            if (fR[z] >= thr) m.set(z);
        s_fgz_lo = m.lo;
        s_fgz_hi = m.hi;
    }
    neighbour_setup(R, row, Dz, bx, xs, ys, fzz, false, nb);
    Mask65 fgz;
    fgz.lo = s_fgz_lo;
    fgz.hi = s_fgz_hi;
    const float seff = s_seff;

    // ---- pass A: first background estimate, counts, recorded frames ------------------------------------------
    double acc[16];
    long long n_over = 0, n_fg_masked = 0, n_fg_nb = 0;
    Mask65 rec;
    rec.clear();
    {
        double sc = 0.0, sb_ = 0.0;
        for (int p = threadIdx.x; p < P; p += NT) {
            const int i = p % bx, j = p / bx;
            const float u1 = u1s[p], u2 = u2s[p];
            O.u1[po + p] = u1;
            O.u2[po + p] = u2;
            const float r2 = u1 * u1 + u2 * u2;
            const bool fg2 = r2 <= kFgR2, ring = r2 >= kBgR2;
            const float bref = bkg_ref(det, xs[i], ys[j]);
            const Mask65 nbm = neighbour_frames(nb, i, j, Dz);
            for (int z = 0; z < Dz; ++z) {
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
                const bool valid = v >= 0.0f, recd = v > -2.5f, over = v == -2.0f;
                const bool fg = fg2 && fgz.get(z);
                const bool nbz = nbm.get(z);
                if (recd) rec.set(z);
                n_over += (over && fg);
                n_fg_masked += (fg && !valid && recd);
                n_fg_nb += (fg && nbz);
                if (valid && !fg && !nbz && ring) {
                    sc += (double)v;
                    sb_ += (double)bref;
                }
            }
        }
        acc[0] = sc;
        acc[1] = sb_;
        acc[2] = (double)n_over;
        acc[3] = (double)n_fg_masked;
        acc[4] = (double)n_fg_nb;
        double a5[5] = {acc[0], acc[1], acc[2], acc[3], acc[4]};
        atomicOr(&s_rec_lo, rec.lo);
        atomicOr(&s_rec_hi, rec.hi);
        block_sum<NT, 5>(a5, red, tot);
        if (threadIdx.x == 0) s_b = (float)tot[0] / fmaxf((float)tot[1], 1e-6f);
        __syncthreads();
        n_over = (long long)tot[2];
        n_fg_masked = (long long)tot[3];
        n_fg_nb = (long long)tot[4];
    }
    // ---- passes B: Poisson-aware clipped background, 4 iterations ----------------------------------------------
    double nbg_d = 0.0;
    for (int it = 0; it < 4; ++it) {
        const float b = s_b;
        double sc = 0.0, sb_ = 0.0;
        for (int p = threadIdx.x; p < P; p += NT) {
            const float u1 = u1s[p], u2 = u2s[p];
            const float r2 = u1 * u1 + u2 * u2;
            if (!(r2 >= kBgR2)) continue;           // background only outside BG_R (r2 >= 12.25 implies not fg2)
            const int i = p % bx, j = p / bx;
            const float bref = bkg_ref(det, xs[i], ys[j]);
            const float bp = b * bref;
            const float thr = (bp + 3.0f * sqrtf(gain * fmaxf(bp, 0.5f))) + 1.0f;
            const Mask65 nbm = neighbour_frames(nb, i, j, Dz);
            for (int z = 0; z < Dz; ++z) {
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
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
    // ---- pass C: summation, centroid, moments, projected spot, per-frame net ---------------------------------
    for (int q = 0; q < 16; ++q) acc[q] = 0.0;
    double nfg = 0.0;
    for (int z = threadIdx.x; z < Dz; z += NT)
        for (int w = 0; w < NT / 32; ++w) fzw[w][z] = 0.0f;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int n_iter = (P + NT - 1) / NT;
    for (int q = 0; q < n_iter; ++q) {
        const int p = threadIdx.x + q * NT;
        const bool have = p < P;
        const int i = have ? p % bx : 0, j = have ? p / bx : 0;
        float u1 = 0.f, u2 = 0.f, bref = 1.f;
        if (have) {
            u1 = u1s[p];
            u2 = u2s[p];
            bref = bkg_ref(det, xs[i], ys[j]);
        }
        const float r2 = u1 * u1 + u2 * u2;
        const bool fg2 = have && r2 <= kFgR2;
        const float bpix = b * bref;
        const float x = xs[i], y = ys[j];
        const float eps1 = u1 * seff, eps2 = u2 * seff;
        const float e12 = eps1 * eps1 + eps2 * eps2;
        Mask65 nbm;
        nbm.clear();
        if (have) nbm = neighbour_frames(nb, i, j, Dz);
        double img2 = 0.0;
        bool okall = true;
        for (int z = 0; z < Dz; ++z) {
            float fzc = 0.0f;
            if (have) {
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
                const bool valid = v >= 0.0f;
                const float c = valid ? v : 0.0f;
                const bool fgzz = fgz.get(z);
                const bool nbz = nbm.get(z);
                const bool clean = valid && !nbz;
                const float net = c - bpix;
                if (fg2 && fgzz && clean) {            // fgv: foreground, valid, not a neighbour's
                    nfg += 1.0;
                    acc[0] += (double)bref;            // sfb
                    acc[1] += (double)net;             // isum
                    acc[2] += (double)c;               // vsum counts
                    acc[3] += (double)bpix;            // vsum0
                    const float wpos = fmaxf(net, 0.0f);
                    acc[4] += (double)wpos;            // sw
                    acc[5] += (double)(wpos * x);
                    acc[6] += (double)(wpos * y);
                    acc[7] += (double)(wpos * fzz[z]);
                    acc[8] += (double)net;             // sws
                    acc[9] += (double)(net * eps1);
                    acc[10] += (double)(net * eps2);
                    acc[11] += (double)(net * e12);
                    const float e3 = fe3[z];
                    acc[12] += (double)(net * e3);
                    acc[13] += (double)(net * (e3 * e3));
                }
                if (fgzz) {
                    if (clean) img2 += (double)net;
                    else okall = false;
                }
                if (fg2 && clean) fzc = net;
            }
            fzc = warp_sumf(fzc);
            if (lane == 0) fzw[wid][z] += fzc;
        }
        if (have) {
            O.img2[po + p] = (float)img2;
            O.all_valid2[po + p] = okall ? 1 : 0;
        }
    }
    double a15[15];
    for (int q = 0; q < 14; ++q) a15[q] = acc[q];
    a15[14] = nfg;
    block_sum<NT, 15>(a15, red, tot);
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
    }
}

// ==================================================================================================================
// pass 2
// ==================================================================================================================
template <int NT>
__global__ void __launch_bounds__(NT) k_pass2(XiDetector det, XiRows R, XiBlock B, const float* __restrict__ arena,
                                              const float* __restrict__ prof, XiPass2In I2, XiPass2Out O,
                                              const int32_t* __restrict__ order, int max_bx, int max_dz,
                                              int* status) {
    extern __shared__ float dyn[];
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

    const int row = order ? order[blockIdx.x] : blockIdx.x;
    const int Dz = R.Dz[row], bx = R.bx[row];
    if (Dz < 1 || Dz > max_dz || bx < 3 || bx > max_bx) {
        if (threadIdx.x == 0) atomicOr(status, 1);
        return;
    }
    const int P = bx * bx;
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
    const float* prof_r = prof + (size_t)R.region[row] * XI_GRID * XI_GRID;
    float* P2s = dyn;               // [P]
    float* P2ps = dyn + P;          // [P] partner
    float* e1s = dyn + 2 * P;       // [P] partner geometry scratch
    float* e2s = dyn + 3 * P;       // [P]
    float* Jps = dyn + 4 * P;       // [P]

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
    for (int z = threadIdx.x; z < Dz; z += NT) {
        float lo, hi;
        bin_limits(iz0, fb, z, B.frames_phi0, B.osc, &lo, &hi);
        fR[z] = rocking_fraction(lo, hi, phi, zeta, B.sm, B.rcw);
        fRp[z] = has_p ? rocking_fraction(lo, hi, R.pphi[row], s_zetap, B.sm, B.rcw) : 0.0f;
    }
    if (has_p) {
        float e1[3] = {s_e1[0], s_e1[1], s_e1[2]}, e2[3] = {s_e2[0], s_e2[1], s_e2[2]};
        float S[3] = {s_S[0], s_S[1], s_S[2]};
        box_geometry(det, S, e1, e2, bx, xs, ys, B.sd, e1s, e2s, nullptr, Jps, &s_seffp);
    }
    __syncthreads();
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
    neighbour_setup(R, row, Dz, bx, xs, ys, fzz, has_p, nb);
    const float pthr = 0.01f * s_pmax;
    const float ppthr = 0.01f * fmaxf(s_ppmax, 1e-12f);

    // ---- pass U: use mask, initial intensity ---------------------------------------------------------------
    // per-thread pixels (at most ceil(97^2 / NT)); use masks are recomputed per pass (cheap) to spare registers
    double acc[16];
    {
        double s_net = 0.0, s_w = 0.0;
        for (int p = threadIdx.x; p < P; p += NT) {
            const int i = p % bx, j = p / bx;
            const float bref = bkg_ref(det, xs[i], ys[j]);
            const float bpix = bg * bref;
            const float P2 = P2s[p], P2p = P2ps[p];
            const Mask65 nbm = neighbour_frames(nb, i, j, Dz);
            for (int z = 0; z < Dz; ++z) {
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
                if (!(v >= 0.0f) || nbm.get(z)) continue;
                const float pv = P2 * fR[z];
                const float ppv = (P2p * fRp[z]) * hp;
                if (!(pv > pthr || ppv > ppthr)) continue;
                s_net += (double)(v - bpix);
                s_w += (double)(pv + ppv);
            }
        }
        double a2[2] = {s_net, s_w};
        block_sum<NT, 2>(a2, red, tot);
        if (threadIdx.x == 0) {
            const float I0 = (float)tot[0] / fmaxf((float)tot[1], 1e-6f);
            s_I = I0;
            s_Ip = I0 * hp;
        }
        __syncthreads();
    }
    // ---- IRLS: Poisson-weighted 2x2 normal equations, float64 sums, N_IRLS iterations ----------------------
    double a11 = 0.0, a12 = 0.0, a22 = 1.0, b1 = 0.0, b2 = 0.0, det2 = 1.0;
    float Iw = 0.0f, Ipw = 0.0f;        // intensities of the last iteration's weights (the variance tail uses them)
    for (int it = 0; it < kIrls; ++it) {
        const float I = s_I, Ip = s_Ip;
        Iw = I;
        Ipw = Ip;
        const float Ipos = fmaxf(I, 0.0f), Ippos = fmaxf(Ip, 0.0f);
        double s11 = 0.0, s1 = 0.0, s12 = 0.0, s22 = 0.0, s2 = 0.0;
        for (int p = threadIdx.x; p < P; p += NT) {
            const int i = p % bx, j = p / bx;
            const float bref = bkg_ref(det, xs[i], ys[j]);
            const float bpix = bg * bref;
            const float P2 = P2s[p], P2p = P2ps[p];
            const Mask65 nbm = neighbour_frames(nb, i, j, Dz);
            for (int z = 0; z < Dz; ++z) {
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
                if (!(v >= 0.0f) || nbm.get(z)) continue;
                const float pv = P2 * fR[z];
                const float ppv = (P2p * fRp[z]) * hp;
                if (!(pv > pthr || ppv > ppthr)) continue;
                const float net = v - bpix;
                float mu = bpix + Ipos * pv;
                if (has_p) mu = mu + Ippos * ppv;
                const float iv = 1.0f / (gain * fmaxf(mu, kVarFloor));
                const float wpp = pv * pv, wpn = pv * net;
                s11 += (double)(wpp * iv);
                s1 += (double)(wpn * iv);
                if (has_p) {
                    s12 += (double)((pv * ppv) * iv);
                    s22 += (double)((ppv * ppv) * iv);
                    s2 += (double)((ppv * net) * iv);
                }
            }
        }
        double a5[5] = {s11, s1, s12, s22, s2};
        block_sum<NT, 5>(a5, red, tot);
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
        det2 = fmax(a11 * a22 - a12 * a12, 1e-30);
        if (threadIdx.x == 0) {
            s_I = (float)((a22 * b1 - a12 * b2) / det2);
            s_Ip = (float)((a11 * b2 - a12 * b1) / det2 * (double)hp);
        }
        __syncthreads();
    }
    const float I = s_I, Ip = s_Ip;
    const float Ippos = fmaxf(Ip, 0.0f);
    const float Iwpos = fmaxf(Iw, 0.0f), Ipwpos = fmaxf(Ipw, 0.0f);
    // ---- tail pass 1: C, a110, C0 (last iteration's weights), use counts, sums for pm / nm, p_valid, p_total, p_fg
    {
        Mask65 fgz;
        fgz.lo = s_fgz_lo;
        fgz.hi = s_fgz_hi;
        for (int q = 0; q < 16; ++q) acc[q] = 0.0;
        for (int p = threadIdx.x; p < P; p += NT) {
            const int i = p % bx, j = p / bx;
            const float bref = bkg_ref(det, xs[i], ys[j]);
            const float bpix = bg * bref;
            const float iv0 = 1.0f / (gain * fmaxf(bpix, kVarFloor));
            const float P2 = P2s[p], P2p = P2ps[p];
            const float u1 = I2.u1[po + p], u2 = I2.u2[po + p];
            const bool fg2 = (u1 * u1 + u2 * u2) <= kFgR2;
            const Mask65 nbm = neighbour_frames(nb, i, j, Dz);
            for (int z = 0; z < Dz; ++z) {
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
                const float pv = P2 * fR[z];
                const float ppv = (P2p * fRp[z]) * hp;
                const bool valid = v >= 0.0f, nbz = nbm.get(z);
                acc[5] += (double)pv;                                       // p_total
                if (valid && !nbz) acc[6] += (double)pv;                    // p_valid
                if (fg2 && fgz.get(z)) acc[7] += (double)pv;                // p_fg numerator
                if (!valid || nbz || !(pv > pthr || ppv > ppthr)) continue;
                const float net = v - bpix;
                float mu = bpix + Iwpos * pv;
                if (has_p) mu = mu + Ipwpos * ppv;
                const float iv = 1.0f / (gain * fmaxf(mu, kVarFloor));
                const float wb = pv * bref;
                acc[0] += (double)(wb * iv);                                // C
                acc[1] += (double)((pv * pv) * iv0);                        // a110
                acc[2] += (double)(wb * iv0);                               // C0
                acc[3] += 1.0;                                              // n use
                acc[4] += (double)pv;                                       // sum wp
                const float resid = has_p ? net - Ippos * ppv : net;
                acc[8] += (double)resid;
            }
        }
        double a9[9];
        for (int q = 0; q < 9; ++q) a9[q] = acc[q];
        block_sum<NT, 9>(a9, red, tot);
    }
    const double Cc = tot[0], a110 = fmax(tot[1], 1e-12), C0 = tot[2];
    const float nuse = (float)tot[3];
    const float pm = (float)tot[4] / fmaxf(nuse, 1.0f);
    const float nm = (float)tot[8] / fmaxf(nuse, 1.0f);
    const float p_total = (float)tot[5], p_valid = (float)tot[6], p_fgn = (float)tot[7];
    // ---- tail pass 2: profile / residual correlation -----------------------------------------------------------
    {
        double sdd = 0.0, spp = 0.0, snn = 0.0;
        for (int p = threadIdx.x; p < P; p += NT) {
            const int i = p % bx, j = p / bx;
            const float bref = bkg_ref(det, xs[i], ys[j]);
            const float bpix = bg * bref;
            const float P2 = P2s[p], P2p = P2ps[p];
            const Mask65 nbm = neighbour_frames(nb, i, j, Dz);
            for (int z = 0; z < Dz; ++z) {
                const float v = sb[(size_t)z * P + p] - R.sb_bias;
                if (!(v >= 0.0f) || nbm.get(z)) continue;
                const float pv = P2 * fR[z];
                const float ppv = (P2p * fRp[z]) * hp;
                if (!(pv > pthr || ppv > ppthr)) continue;
                const float net = v - bpix;
                const float resid = has_p ? net - Ippos * ppv : net;
                const float dp = pv - pm, dn = resid - nm;
                sdd += (double)(dp * dn);
                spp += (double)(dp * dp);
                snn += (double)(dn * dn);
            }
        }
        double a3[3] = {sdd, spp, snn};
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

__global__ void k_gather(XiFrames F, XiGatherRows G, float* __restrict__ arena, int32_t* __restrict__ cnt,
                         const int32_t* __restrict__ order) {
    const int row = order ? order[blockIdx.x] : blockIdx.x;
    const int iz0 = G.iz0[row], fb = G.fb[row], Dz = G.Dz[row], bx = G.bx[row];
    const int s = G.pxs ? G.pxs[row] : 1;
    const int ix0 = G.ix0[row], iy0 = G.iy0[row];
    const int P = bx * bx;
    const int span = Dz * fb;
    const int w0 = max(0, iz0 - F.first_fi), w1 = min(F.n_frames, iz0 + span - F.first_fi);
    float* dst = arena + G.sb_off[row];
    const size_t fstride = (size_t)F.ny * F.nx * (F.is_float ? sizeof(float) : sizeof(uint32_t));
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

__global__ void k_decode_bins(XiGatherRows G, float* __restrict__ arena, const int32_t* __restrict__ cnt) {
    const int row = blockIdx.x;
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

size_t pass1_smem(int max_bx) { return (size_t)2 * max_bx * max_bx * sizeof(float); }
size_t pass2_smem(int max_bx) { return (size_t)5 * max_bx * max_bx * sizeof(float); }

int rows_check(const XiRows* R) {
    if (!R) return fail(XI_E_ARG, "rows: null");
    if (R->n < 0 || (R->order && R->n_order < 0)) return fail(XI_E_ARG, "rows: negative count");
    if (R->K < 0 || R->K > XI_MAX_K) return fail(XI_E_LIMIT, "rows: neighbour columns beyond XI_MAX_K");
    if (R->max_bx < 3 || R->max_bx > XI_MAX_BX || R->max_dz < 1 || R->max_dz > XI_MAX_DZ)
        return fail(XI_E_LIMIT, "rows: max_bx / max_dz outside 3..97 / 1..65");
    return XI_OK;
}

template <int NT>
int launch_pass1(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena,
                        XiPass1Out* O, cudaStream_t s, int nblk) {
    size_t sm = pass1_smem(R->max_bx);
    cudaFuncSetAttribute(k_pass1<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_pass1<NT><<<nblk, NT, sm, s>>>(*det, *R, *B, arena, *O, R->order, R->max_bx, R->max_dz, status_ptr());
    return cuda_check("xi_pass1");
}

template <int NT>
int launch_pass2(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena,
                        const float* prof, const XiPass2In* in, XiPass2Out* O, cudaStream_t s, int nblk) {
    size_t sm = pass2_smem(R->max_bx);
    cudaFuncSetAttribute(k_pass2<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_pass2<NT><<<nblk, NT, sm, s>>>(*det, *R, *B, arena, prof, *in, *O, R->order, R->max_bx, R->max_dz,
                                     status_ptr());
    return cuda_check("xi_pass2");
}

}  // namespace

// ==================================================================================================================
// C ABI
// ==================================================================================================================
extern "C" {

const char* xi_last_error(void) { return g_err; }

int xi_version(void) { return 1; }

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


int xi_pass1(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena, XiPass1Out* O,
             void* stream) {
    if (!det || !B || !arena || !O) return fail(XI_E_ARG, "xi_pass1: null argument");
    int rc = rows_check(R);
    if (rc) return rc;
    const int nblk = R->order ? R->n_order : R->n;
    if (nblk == 0) return XI_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int P = R->max_bx * R->max_bx;
    if (P <= 96) return launch_pass1<64>(det, R, B, arena, O, s, nblk);
    if (P <= 200) return launch_pass1<128>(det, R, B, arena, O, s, nblk);
    return launch_pass1<256>(det, R, B, arena, O, s, nblk);
}


int xi_pass2(const XiDetector* det, const XiRows* R, const XiBlock* B, const float* arena, const float* prof,
             const XiPass2In* in, XiPass2Out* O, void* stream) {
    if (!det || !B || !arena || !prof || !in || !O) return fail(XI_E_ARG, "xi_pass2: null argument");
    int rc = rows_check(R);
    if (rc) return rc;
    const int nblk = R->order ? R->n_order : R->n;
    if (nblk == 0) return XI_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int P = R->max_bx * R->max_bx;
    if (P <= 96) return launch_pass2<64>(det, R, B, arena, prof, in, O, s, nblk);
    if (P <= 200) return launch_pass2<128>(det, R, B, arena, prof, in, O, s, nblk);
    return launch_pass2<256>(det, R, B, arena, prof, in, O, s, nblk);
}

int xi_gather(const XiFrames* F, const XiGatherRows* G, float* arena, int32_t* cnt, void* stream) {
    if (!F || !G || !arena || !F->data) return fail(XI_E_ARG, "xi_gather: null argument");
    if (F->n_frames < 0 || F->ny <= 0 || F->nx <= 0 || G->n < 0) return fail(XI_E_ARG, "xi_gather: bad sizes");
    const int nblk = G->order ? G->n_order : G->n;
    if (nblk == 0 || F->n_frames == 0) return XI_OK;
    k_gather<<<nblk, 128, 0, (cudaStream_t)stream>>>(*F, *G, arena, cnt, G->order);
    return cuda_check("xi_gather");
}

int xi_decode_bins(const XiGatherRows* G, float* arena, const int32_t* cnt, void* stream) {
    if (!G || !arena || !cnt) return fail(XI_E_ARG, "xi_decode_bins: null argument");
    if (G->n == 0) return XI_OK;
    k_decode_bins<<<G->n, 256, 0, (cudaStream_t)stream>>>(*G, arena, cnt);
    return cuda_check("xi_decode_bins");
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
