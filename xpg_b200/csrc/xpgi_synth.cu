// Device generator of synthetic uint32 frame wedges (the model of xpg_b200/synth.py): flat background with a
// radial ramp, Gaussian spots (tangential / radial widths, frame-integrated Gaussian rocking curve), Poisson noise
// from a counter-based hash of (seed, frame, pixel), module gaps at 0xFFFFFFFF.
//
// The expected counts are built in place: the output wedge is first used as a float32 image (background, then
// spots added with atomics) and each pixel is then replaced by its Poisson draw. No scratch memory.
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

__device__ __forceinline__ bool in_gap(int y, int x, int gaps) {
    if (!gaps) return false;
    if (y >= 195 && ((y - 195) % 212) < 17) return true;
    if (x >= 487 && ((x - 487) % 494) < 7) return true;
    return false;
}

__global__ void k_background(float* __restrict__ img, int n_frames, int ny, int nx, XiSynthBackground bg) {
    const size_t P = (size_t)ny * nx;
    const size_t total = P * n_frames;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i % P;
        const int y = (int)(p / nx), x = (int)(p % nx);
        const double r = hypot(x + 1.0 - bg.orgx, y + 1.0 - bg.orgy);
        img[i] = (float)(bg.level * (1.0 + bg.ramp * r / bg.rmax));
    }
}

// one CTA per spot: every frame of the wedge its rocking curve reaches (|z - zc| < 5 sigma_z), a window of
// +-4.5 radial sigma (4..60 px), 2 x 2 sub-pixel samples
__global__ void k_spots(float* __restrict__ img, int first_frame, int n_frames, int ny, int nx, XiSynthSpots S) {
    const int r = blockIdx.x;
    if (r >= S.n) return;
    const double xc = S.x[r], yc = S.y[r], zc = S.z[r];
    const double st = S.sig_t[r], sr = S.sig_r[r], sz = S.sig_z[r];
    const double counts = S.counts[r];
    double rx = xc - S.orgx, ry = yc - S.orgy;
    const double rn = hypot(rx, ry);
    if (rn > 1e-6) { rx /= rn; ry /= rn; } else { rx = 1.0; ry = 0.0; }
    const int half = min(max((int)ceil(4.5 * sr), 4), 60);
    const int W = 2 * half + 1;
    const int ix = (int)floor(xc - 1.0 + 0.5), iy = (int)floor(yc - 1.0 + 0.5);
    const double norm = 1.0 / (4.0 * 2.0 * 3.141592653589793 * sr * st);
    for (int w = 0; w < n_frames; ++w) {
        const double z0 = first_frame - 1 + w, z1 = z0 + 1.0;
        if (!(zc + 5.0 * sz > z0 && zc - 5.0 * sz < z1)) continue;
        const double fz = 0.5 * (erf((z1 - zc) / (1.4142135623730951 * sz)) - erf((z0 - zc) / (1.4142135623730951 * sz)));
        const double amp = counts * fz * norm;
        float* F = img + (size_t)w * ny * nx;
        for (int q = threadIdx.x; q < W * W; q += blockDim.x) {
            const int px = ix - half + q % W, py = iy - half + q / W;
            if (px < 0 || px >= nx || py < 0 || py >= ny) continue;
            double g = 0.0;
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b) {
                    const double dx = px + 1.0 + (b + 0.5) * 0.5 - 0.5 - xc;
                    const double dy = py + 1.0 + (a + 0.5) * 0.5 - 0.5 - yc;
                    const double ur = dx * rx + dy * ry, ut = -dx * ry + dy * rx;
                    g += exp(-0.5 * ((ur / sr) * (ur / sr) + (ut / st) * (ut / st)));
                }
            atomicAdd(F + (size_t)py * nx + px, (float)(amp * g));
        }
    }
}

__global__ void k_poisson(float* __restrict__ img, int first_frame, int n_frames, int ny, int nx, uint64_t seed,
                          int gaps) {
    const size_t P = (size_t)ny * nx;
    const size_t total = P * n_frames;
    uint32_t* out = reinterpret_cast<uint32_t*>(img);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i % P;
        const int f = first_frame + (int)(i / P);
        const int y = (int)(p / nx), x = (int)(p % nx);
        const double lam = (double)img[i];
        uint32_t k = 0;
        if (in_gap(y, x, gaps)) {
            k = 0xFFFFFFFFu;
        } else {
            const uint64_t h = mix64(seed * 0x9E3779B97F4A7C15ull + ((uint64_t)f << 40) + p);
            const double u = unit_double(h);
            if (lam < 40.0) {
                double pk = exp(-lam), F = pk;
                uint32_t n = 0;
                while (u > F && n < 400) {
                    ++n;
                    pk *= lam / n;
                    F += pk;
                }
                k = n;
            } else {
                const double u2 = unit_double(mix64(h ^ 0xD1B54A32D192ED03ull));
                const double g = sqrt(-2.0 * log(u)) * cos(6.283185307179586 * u2);
                const double v = floor(lam + sqrt(lam) * g + 0.5);
                k = v <= 0.0 ? 0u : (v >= 4294967294.0 ? 0xFFFFFFFEu : (uint32_t)v);
            }
        }
        out[i] = k;
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
    float* img = reinterpret_cast<float*>(out);
    const int grid = 148 * 16;
    k_background<<<grid, 256, 0, s>>>(img, n_frames, ny, nx, *bg);
    if (spots->n > 0) k_spots<<<spots->n, 128, 0, s>>>(img, first_frame, n_frames, ny, nx, *spots);
    k_poisson<<<grid, 256, 0, s>>>(img, first_frame, n_frames, ny, nx, seed, gaps);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof g_err, "xi_synth_frames: %s", cudaGetErrorString(e));
        return XI_E_CUDA;
    }
    return XI_OK;
}

}  // extern "C"
