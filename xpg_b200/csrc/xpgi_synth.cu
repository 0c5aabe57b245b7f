// Device generator of synthetic uint32 frame wedges (the model of xpg_b200/synth.py): flat background with a
// radial ramp, Gaussian spots (tangential / radial widths, frame-integrated Gaussian rocking curve), Poisson noise
// from a counter-based hash of (seed, frame, pixel), module gaps at 0xFFFFFFFF.
//
// Two launches and no scratch memory: every pixel's background draw is written once, then each spot adds its own
// Poisson draw to the pixels of its window (atomics; a sum of independent Poisson draws is the draw of the summed
// mean), so a frame costs one write of the wedge plus the spot windows.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include "xpgi.h"
#include "xpgi_synth.h"

namespace {

thread_local char g_err[256] = {0};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    // splitmix64 finaliser
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

__device__ __forceinline__ double unit_double(uint64_t h) {
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// module gaps: 17-row bands every 212 rows from row 195, 7-column bands every 494 columns from column 487
__device__ __forceinline__ bool gap_row(int y, int gaps) { return gaps && y >= 195 && ((y - 195) % 212) < 17; }
__device__ __forceinline__ bool gap_col(int x, int gaps) { return gaps && x >= 487 && ((x - 487) % 494) < 7; }
__device__ __forceinline__ bool in_gap(int y, int x, int gaps) { return gap_row(y, gaps) || gap_col(x, gaps); }

// Poisson draw of mean lam from one uniform u (inversion for small means, rounded normal approximation above 40,
// with a second uniform from the same hash)
__device__ __forceinline__ uint32_t poisson_draw(float lam, uint64_t h) {
    const float u = (float)unit_double(h);
    if (lam < 40.0f) {
        float pk = __expf(-lam), F = pk;
        uint32_t n = 0;
        while (u > F && n < 400) {
            ++n;
            pk *= lam / (float)n;
            F += pk;
        }
        return n;
    }
    const float u2 = (float)unit_double(mix64(h ^ 0xD1B54A32D192ED03ull));
    const float g = sqrtf(-2.0f * __logf(u)) * __cosf(6.2831853f * u2);
    const float v = floorf(lam + sqrtf(lam) * g + 0.5f);
    return v <= 0.0f ? 0u : (v >= 4294967040.0f ? 0xFFFFFF00u : (uint32_t)v);
}

// background counts of every pixel of the wedge (flat level with a radial ramp), gaps flagged: CTAs stride over
// (detector row, frame), threads over the row's pixels, so that every index is 32-bit arithmetic (the hash key is the
// same 64-bit sum of frame and pixel index as a flat index would give)
__global__ void k_background_counts(uint32_t* __restrict__ out, int first_frame, int n_frames, int ny, int nx,
                                    XiSynthBackground bg, uint64_t seed, int gaps) {
    const float ox = (float)bg.orgx, oy = (float)bg.orgy, lev = (float)bg.level, k = (float)(bg.ramp / bg.rmax);
    for (int f = blockIdx.y; f < n_frames; f += gridDim.y) {
        uint32_t* F = out + (size_t)f * ny * nx;
        const uint64_t fkey = seed * 0x9E3779B97F4A7C15ull + ((uint64_t)(first_frame + f) << 40);
        for (int y = blockIdx.x; y < ny; y += gridDim.x) {
            const size_t row = (size_t)y * nx;
            const bool gy = gap_row(y, gaps);
            const float dy = (float)y + 1.0f - oy;
            for (int x = threadIdx.x; x < nx; x += blockDim.x) {
                uint32_t c;
                if (gy || gap_col(x, gaps)) {
                    c = 0xFFFFFFFFu;
                } else {
                    const float r = hypotf((float)x + 1.0f - ox, dy);
                    c = poisson_draw(lev * (1.0f + k * r), mix64(fkey + row + (size_t)x));
                }
                F[row + x] = c;
            }
        }
    }
}

// spot counts added to the background's: one CTA per spot, every frame of the wedge its rocking curve reaches
// (|z - zc| < 5 sigma_z), a window of +-4.5 radial sigma (4..60 px), 2 x 2 sub-pixel samples of the Gaussian, an
// independent Poisson draw per pixel (the sum of the two draws is the Poisson draw of the summed mean)
__global__ void k_spot_counts(uint32_t* __restrict__ out, int first_frame, int n_frames, int ny, int nx,
                              XiSynthSpots S, uint64_t seed, int gaps) {
    if ((int)blockIdx.x >= S.n) return;
    const int r = S.index ? S.index[blockIdx.x] : (int)blockIdx.x;
    const double xc = S.x[r], yc = S.y[r], zc = S.z[r];
    const double sz = S.sig_z[r];
    const float st = (float)S.sig_t[r], sr = (float)S.sig_r[r];
    double rx = xc - S.orgx, ry = yc - S.orgy;
    const double rn = hypot(rx, ry);
    if (rn > 1e-6) { rx /= rn; ry /= rn; } else { rx = 1.0; ry = 0.0; }
    const float frx = (float)rx, fry = (float)ry;
    const int half = min(max((int)ceil(4.5 * (double)sr), 4), 60);
    const int W = 2 * half + 1;
    const int ix = (int)floor(xc - 1.0 + 0.5), iy = (int)floor(yc - 1.0 + 0.5);
    const float fxc = (float)(xc - ix), fyc = (float)(yc - iy);       // centre relative to the middle pixel's index
    const double norm = 1.0 / (4.0 * 2.0 * 3.141592653589793 * (double)sr * (double)st);
    const uint64_t salt = seed * 0xC2B2AE3D27D4EB4Full + (uint64_t)r * 0x165667B19E3779F9ull;
    for (int w = 0; w < n_frames; ++w) {
        const double z0 = first_frame - 1 + w, z1 = z0 + 1.0;
        if (!(zc + 5.0 * sz > z0 && zc - 5.0 * sz < z1)) continue;
        const double fz = 0.5 * (erf((z1 - zc) / (1.4142135623730951 * sz)) - erf((z0 - zc) / (1.4142135623730951 * sz)));
        const float amp = (float)(S.counts[r] * fz * norm);
        if (!(amp > 0.0f)) continue;
        uint32_t* F = out + (size_t)w * ny * nx;
        for (int q = threadIdx.x; q < W * W; q += blockDim.x) {
            const int dxp = q % W - half, dyp = q / W - half;
            const int px = ix + dxp, py = iy + dyp;
            if (px < 0 || px >= nx || py < 0 || py >= ny || in_gap(py, px, gaps)) continue;
            float g = 0.0f;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    // pixel (ix + dxp) spans coordinates ix + dxp + 0.5 .. + 1.5; sub-sample centres at +-0.25
                    const float dx = (float)dxp + (1.0f - fxc) + ((b + 0.5f) * 0.5f - 0.5f);
                    const float dy = (float)dyp + (1.0f - fyc) + ((a + 0.5f) * 0.5f - 0.5f);
                    const float ur = dx * frx + dy * fry, ut = -dx * fry + dy * frx;
                    g += __expf(-0.5f * ((ur / sr) * (ur / sr) + (ut / st) * (ut / st)));
                }
            const float lam = amp * g;
            if (lam < 1e-7f) continue;
            const uint32_t c = poisson_draw(lam, mix64(salt + ((uint64_t)(first_frame + w) << 40) +
                                                        (uint64_t)py * nx + px));
            if (c) atomicAdd(F + (size_t)py * nx + px, c);
        }
    }
}

}  // namespace

extern "C" {

const char* xi_synth_last_error(void) { return g_err; }

int xi_synth_frames(const XiSynthSpots* spots, const XiSynthBackground* bg, int first_frame, int n_frames, int ny,
                    int nx, uint64_t seed, int gaps, uint32_t* out, void* stream) {
    if (!spots || !bg || !out || n_frames < 0 || ny <= 0 || nx <= 0) {
        snprintf(g_err, sizeof g_err, "xi_synth_frames: bad argument");
        return XI_E_ARG;
    }
    if (n_frames == 0) return XI_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid((unsigned)(ny < 296 ? ny : 296), (unsigned)(n_frames < 32 ? n_frames : 32));
    k_background_counts<<<grid, 256, 0, s>>>(out, first_frame, n_frames, ny, nx, *bg, seed, gaps);
    if (spots->n > 0) k_spot_counts<<<spots->n, 128, 0, s>>>(out, first_frame, n_frames, ny, nx, *spots, seed, gaps);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof g_err, "xi_synth_frames: %s", cudaGetErrorString(e));
        return XI_E_CUDA;
    }
    return XI_OK;
}

}  // extern "C"
