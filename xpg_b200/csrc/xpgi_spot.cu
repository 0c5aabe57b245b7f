// Strong-pixel classifier of spot finding (include/xpgi.h, "Spot finding"): XPG's dispersion test and its extended
// second pass (xpg/spotfind.py:27-97) on float32 frames, bit for bit. A CTA takes a 32 x 8 tile of one frame: the
// window sums of the valid-pixel count, the values and their squares are separable, so the tile and its halo are
// staged in shared memory, summed along x for every staged row, then along y for every output pixel, each sum over
// its window in increasing coordinate from zero (the order the reference's pooling sums in; zero outside the frame).
// Three launches per call: the dispersion test (first-pass strong mask and local mean), the background pixels of the
// extended pass, the extended pass itself.
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpgi.h"
#include "xpgi_internal.h"

namespace {

constexpr int kTW = 32, kTH = 8, kNT = kTW * kTH;
constexpr float kDispersionSigmaB = 6.0f;

// window sums of (w, x, x * x) of this thread's pixel, x = w ? value : 0, w from the source's rule; hx, hy: half widths
struct Sums {
    float n, s1, s2;
};

template <class Src>
__device__ Sums tile_sums(const Src& src, int b, int ny, int nx, int hx, int hy, float* sm) {
    const int W = kTW + 2 * hx, H = kTH + 2 * hy;
    float* tw = sm;                   // staged weights, H x W
    float* tx = tw + H * W;           // staged values
    float* hw = tx + H * W;           // sums along x, H x kTW
    float* hs = hw + H * kTW;
    float* hq = hs + H * kTW;
    const int x0 = blockIdx.x * kTW - hx, y0 = blockIdx.y * kTH - hy;
    for (int i = threadIdx.x; i < H * W; i += kNT) {
        const int r = i / W, c = i % W;
        const int y = y0 + r, x = x0 + c;
        float w = 0.0f, v = 0.0f;
        if (y >= 0 && y < ny && x >= 0 && x < nx) src.load(b, y, x, w, v);
        tw[i] = w;
        tx[i] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < H * kTW; i += kNT) {
        const int r = i / kTW, c = i % kTW;
        float a = 0.0f, s = 0.0f, q = 0.0f;
        for (int d = 0; d <= 2 * hx; ++d) {
            const float v = tx[r * W + c + d];
            a = a + tw[r * W + c + d];
            s = s + v;
            q = q + v * v;
        }
        hw[i] = a;
        hs[i] = s;
        hq[i] = q;
    }
    __syncthreads();
    const int r = threadIdx.x / kTW, c = threadIdx.x % kTW;
    Sums o{0.0f, 0.0f, 0.0f};
    for (int d = 0; d <= 2 * hy; ++d) {
        const int k = (r + d) * kTW + c;
        o.n = o.n + hw[k];
        o.s1 = o.s1 + hs[k];
        o.s2 = o.s2 + hq[k];
    }
    return o;
}

// a frame's pixels entering the window sums: the valid ones (value >= 0), or those whose flag in sel is set
struct FrameSrc {
    const float* img;
    const uint8_t* sel;
    int ny, nx;
    __device__ void load(int b, int y, int x, float& w, float& v) const {
        const size_t k = ((size_t)b * ny + y) * nx + x;
        const float p = img[k];
        const bool on = sel ? sel[k] != 0 : p >= 0.0f;
        w = on ? 1.0f : 0.0f;
        v = on ? p : 0.0f;
    }
};

__device__ bool any_flag(const uint8_t* f, int b, int ny, int nx, int y, int x, int r) {
    for (int dy = -r; dy <= r; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= ny) continue;
        for (int dx = -r; dx <= r; ++dx) {
            const int xx = x + dx;
            if (xx >= 0 && xx < nx && f[((size_t)b * ny + yy) * nx + xx]) return true;
        }
    }
    return false;
}

// the dispersion test (xpg/spotfind.py:41-54): first-pass strong mask and local mean
__global__ void __launch_bounds__(kNT) k_spot_dispersion(const float* __restrict__ img, int ny, int nx, int hx,
                                                         int hy, float gain, float n_s, float min_local,
                                                         uint8_t* __restrict__ s1, float* __restrict__ mean1) {
    extern __shared__ float sm[];
    const int b = blockIdx.z;
    FrameSrc src{img, nullptr, ny, nx};
    const Sums t = tile_sums(src, b, ny, nx, hx, hy, sm);
    const int y = blockIdx.y * kTH + threadIdx.x / kTW, x = blockIdx.x * kTW + threadIdx.x % kTW;
    if (y >= ny || x >= nx) return;
    const size_t k = ((size_t)b * ny + y) * nx + x;
    const float p = img[k];
    const bool valid = p >= 0.0f;
    const float xv = valid ? p : 0.0f;
    const float nn = fmaxf(t.n, 2.0f);
    const float mean = t.s1 / nn;
    const float var = fmaxf((t.s2 - t.s1 * mean) / (nn - 1.0f), 0.0f);
    const float thr = gain * (1.0f + kDispersionSigmaB * sqrtf(2.0f / (nn - 1.0f)));
    const bool disp = var > thr * fmaxf(mean, 1e-6f);
    const bool strong = (xv - mean) > n_s * sqrtf(gain * fmaxf(mean, 1.0f));
    s1[k] = (valid && t.n >= min_local && disp && strong) ? 1 : 0;
    mean1[k] = mean;
}

// background pixels of the extended pass (xpg/spotfind.py:78-79): valid, not within 1 px of first-pass signal, at
// most mean + background_pixel x sigma
__global__ void __launch_bounds__(256) k_spot_background(const float* __restrict__ img, int n_frames, int ny, int nx,
                                                          const uint8_t* __restrict__ s1,
                                                          const float* __restrict__ mean1, float gain, float bgp,
                                                          uint8_t* __restrict__ bg) {
    const int64_t k = (int64_t)blockIdx.x * 256 + threadIdx.x;
    const int64_t n = (int64_t)n_frames * ny * nx;
    if (k >= n) return;
    const int x = (int)(k % nx), y = (int)((k / nx) % ny), b = (int)(k / ((int64_t)nx * ny));
    const float p = img[k];
    const float m = mean1[k];
    const float sig1 = sqrtf(gain * fmaxf(m, 0.5f));
    bg[k] = (p >= 0.0f && !any_flag(s1, b, ny, nx, y, x, 1) && p <= m + bgp * sig1) ? 1 : 0;
}

// the extended pass (xpg/spotfind.py:80-91): the background re-estimated over the wider window of background pixels;
// a pixel within 2 px of first-pass signal is strong when it exceeds it by signal_pixel sigma
__global__ void __launch_bounds__(kNT) k_spot_extended(const float* __restrict__ img, int ny, int nx, int hx, int hy,
                                                       float gain, float sp, float min_local4,
                                                       const uint8_t* __restrict__ bg, const uint8_t* __restrict__ s1,
                                                       uint8_t* __restrict__ strong, float* __restrict__ mean_out) {
    extern __shared__ float sm[];
    const int b = blockIdx.z;
    FrameSrc src{img, bg, ny, nx};
    const Sums t = tile_sums(src, b, ny, nx, hx, hy, sm);
    const int y = blockIdx.y * kTH + threadIdx.x / kTW, x = blockIdx.x * kTW + threadIdx.x % kTW;
    if (y >= ny || x >= nx) return;
    const size_t k = ((size_t)b * ny + y) * nx + x;
    const float p = img[k];
    const float nn = fmaxf(t.n, 2.0f);
    const float mean = t.s1 / nn;
    const float var = fmaxf((t.s2 - t.s1 * mean) / (nn - 1.0f), 0.0f);
    const float sig = sqrtf(fmaxf(gain * fmaxf(mean, 0.5f), var));
    const bool st = p >= 0.0f && t.n >= min_local4 && (p - mean) > sp * sig;
    strong[k] = (st && any_flag(s1, b, ny, nx, y, x, 2)) ? 1 : 0;
    mean_out[k] = mean;
}

size_t tile_smem(int hx, int hy) {
    const size_t W = kTW + 2 * hx, H = kTH + 2 * hy;
    return (2 * H * W + 3 * H * kTW) * sizeof(float);
}

}  // namespace

extern "C" size_t xi_spot_workspace(int n_frames, int ny, int nx) {
    if (n_frames < 0 || ny < 0 || nx < 0) return 0;
    const size_t n = (size_t)n_frames * ny * nx;
    return ((n + 255) / 256 * 256) * 2 + n * sizeof(float);
}

extern "C" int xi_spot_strong(const float* img, int n_frames, int ny, int nx, float gain, const XiSpotParams* p,
                              uint8_t* strong, float* mean, void* ws, size_t ws_bytes, void* stream) {
    if (!p || n_frames < 0 || ny < 0 || nx < 0) return xi_fail(XI_E_ARG, "xi_spot_strong: null argument or size");
    const size_t n = (size_t)n_frames * ny * nx;
    if (n == 0) return XI_OK;
    if (!img || !strong || !mean) return xi_fail(XI_E_ARG, "xi_spot_strong: null pointer");
    if (p->nbx < 0 || p->nby < 0 || p->nbx > XI_SPOT_MAX_HALF || p->nby > XI_SPOT_MAX_HALF)
        return xi_fail(XI_E_LIMIT, "xi_spot_strong: window half-size beyond XI_SPOT_MAX_HALF");
    if (n_frames > 65535) return xi_fail(XI_E_LIMIT, "xi_spot_strong: more than 65535 frames in one call");
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid((unsigned)((nx + kTW - 1) / kTW), (unsigned)((ny + kTH - 1) / kTH), (unsigned)n_frames);
    const float ml = (float)p->min_local;
    if (!p->extended) {
        k_spot_dispersion<<<grid, kNT, tile_smem(p->nbx, p->nby), s>>>(img, ny, nx, p->nbx, p->nby, gain,
                                                                       p->signal_pixel, ml, strong, mean);
        return xi_cuda_check("xi_spot_strong");
    }
    if (!ws || ws_bytes < xi_spot_workspace(n_frames, ny, nx)) return xi_fail(XI_E_ARG, "xi_spot_strong: workspace");
    uint8_t* s1 = static_cast<uint8_t*>(ws);
    uint8_t* bg = s1 + (n + 255) / 256 * 256;
    float* mean1 = reinterpret_cast<float*>(bg + (n + 255) / 256 * 256);
    const int hx2 = 2 * p->nbx + 1, hy2 = 2 * p->nby + 1;
    const size_t sm2 = tile_smem(hx2, hy2);
    if (sm2 > 48 * 1024) cudaFuncSetAttribute(k_spot_extended, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
    k_spot_dispersion<<<grid, kNT, tile_smem(p->nbx, p->nby), s>>>(img, ny, nx, p->nbx, p->nby, gain,
                                                                   p->signal_pixel, ml, s1, mean1);
    k_spot_background<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(img, n_frames, ny, nx, s1, mean1, gain,
                                                                  p->background_pixel, bg);
    k_spot_extended<<<grid, kNT, sm2, s>>>(img, ny, nx, hx2, hy2, gain, p->signal_pixel, 4.0f * ml, bg, s1, strong,
                                           mean);
    return xi_cuda_check("xi_spot_strong");
}
