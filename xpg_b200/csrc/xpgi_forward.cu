// Forward-model likelihood passes (XPG's pixel-level forward integrator, xpg/forward/): the fused scatter / gather
// of the separable profile factors of reflections' boxes into / from a dense window of voxels, the work of
// xpg/forward/kernels.py:34-103 (Triton) and of the eager passes WindowModel.mu / grad_ratio / grad_newton
// (xpg/forward/model.py:476-577).
//
// One CTA per reflection of the chunk: its threads take the box's pixels, each forms f = sum_t R[t, row, z] *
// P[t, row, y, x] for every frame z of the box (the row's P stays in L1 across the frames), and either adds
// I f + beta to the window voxel (scatter: float atomics, several reflections share voxels) or accumulates the
// weighted sums of the row in float64 (gather), reduced over the CTA and added once to the row's output.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "xpgi.h"

namespace {

thread_local char g_err[256] = {0};

int fm_fail(int code, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

struct Box {
    int64_t kz0, ky0, kx0;      // window coordinates of the box origin
};

__device__ __forceinline__ Box box_origin(const XiFmBoxes& B, const XiFmWindow& W, int row) {
    Box o;
    o.kz0 = B.iz0[row] - W.f0;
    o.ky0 = B.iy0[row] - W.y0;
    o.kx0 = B.ix0[row] - W.x0;
    return o;
}

// f of pixel p (y * b + x) of the row's box on frame z: the terms' products rounded, then summed in term order
__device__ __forceinline__ float fraction(const XiFmBoxes& B, int row, int z, int p) {
    const size_t bb = (size_t)B.b * B.b;
    float f = 0.0f;
    for (int t = 0; t < B.n_terms; ++t) {
        const float r = __ldg(B.R + ((size_t)t * B.n + row) * B.Dz + z);
        const float g = r * __ldg(B.P + ((size_t)t * B.n + row) * bb + p);
        f = t == 0 ? g : f + g;
    }
    return f;
}

__global__ void k_fm_scatter(XiFmBoxes B, XiFmWindow W, const float* __restrict__ I, const float* __restrict__ beta,
                             float* __restrict__ mu) {
    const int row = blockIdx.x;
    const Box o = box_origin(B, W, row);
    const float Ir = I[row];
    const float br = beta ? beta[row] : 0.0f;
    const int bb = B.b * B.b;
    for (int z = 0; z < B.Dz; ++z) {
        const int64_t kz = o.kz0 + z;
        if (kz < 0 || kz >= W.nf) continue;
        for (int p = threadIdx.x; p < bb; p += blockDim.x) {
            const int64_t ky = o.ky0 + p / B.b, kx = o.kx0 + p % B.b;
            if (ky < 0 || ky >= W.ny || kx < 0 || kx >= W.nx) continue;
            float val = fraction(B, row, z, p) * Ir;
            if (beta) val = val + br;
            atomicAdd(mu + (kz * W.ny + ky) * W.nx + kx, val);
        }
    }
}

template <typename NST>
__device__ __forceinline__ float ns_value(const void* NS, int64_t v) {
    return (float)reinterpret_cast<const NST*>(NS)[v];
}

template <typename NST, int MODE>
__global__ void k_fm_gather(XiFmBoxes B, XiFmWindow W, const int64_t* __restrict__ rows, const float* __restrict__ A,
                            const float* __restrict__ M, const void* __restrict__ NS, float* __restrict__ g,
                            float* __restrict__ fd) {
    const int row = blockIdx.x;
    const Box o = box_origin(B, W, row);
    const int bb = B.b * B.b;
    double acc = 0.0, accd = 0.0;
    for (int z = 0; z < B.Dz; ++z) {
        const int64_t kz = o.kz0 + z;
        if (kz < 0 || kz >= W.nf) continue;
        for (int p = threadIdx.x; p < bb; p += blockDim.x) {
            const int64_t ky = o.ky0 + p / B.b, kx = o.kx0 + p % B.b;
            if (ky < 0 || ky >= W.ny || kx < 0 || kx >= W.nx) continue;
            const int64_t v = (kz * W.ny + ky) * W.nx + kx;
            const float ns = ns_value<NST>(NS, v);
            if (!(ns >= 0.0f)) continue;
            const float f = fraction(B, row, z, p);
            const float m = M[v];
            if (MODE == 0) {
                acc += (double)(f * (A[v] / m));
            } else {
                acc += (double)(f * (1.0f - fmaxf(ns, 0.0f) / m));
                accd += (double)((f * f) / fmaxf(m, 1e-6f));
            }
        }
    }
    __shared__ double s_acc[2][32];
    for (int off = 16; off > 0; off >>= 1) {
        acc += __shfl_down_sync(0xffffffffu, acc, off);
        accd += __shfl_down_sync(0xffffffffu, accd, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_acc[0][warp] = acc;
        s_acc[1][warp] = accd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, d = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += s_acc[0][w];
            d += s_acc[1][w];
        }
        const int64_t r = rows ? rows[row] : row;
        atomicAdd(g + r, (float)a);
        if (MODE == 1) atomicAdd(fd + r, (float)d);
    }
}

int check_boxes(const XiFmBoxes* B, const XiFmWindow* W) {
    if (!B || !W) return fm_fail(XI_E_ARG, "forward pass: null argument");
    if (B->n < 0 || B->n_terms < 1 || B->n_terms > 4 || B->Dz < 1 || B->b < 1)
        return fm_fail(XI_E_ARG, "forward pass: bad box shape (n >= 0, 1..4 terms, Dz >= 1, b >= 1)");
    if (B->n > 0 && (!B->R || !B->P || !B->iz0 || !B->iy0 || !B->ix0))
        return fm_fail(XI_E_ARG, "forward pass: null factor or origin array");
    if (W->nf < 0 || W->ny < 0 || W->nx < 0) return fm_fail(XI_E_ARG, "forward pass: negative window size");
    return XI_OK;
}

int launch_check(const char* who) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof g_err, "%s: %s", who, cudaGetErrorString(e));
        return XI_E_CUDA;
    }
    return XI_OK;
}

constexpr int kFmThreads = 128;

template <typename NST>
void launch_gather(const XiFmBoxes& B, const XiFmWindow& W, const int64_t* rows, const float* A, const float* M,
                   const void* NS, int mode, float* g, float* fd, cudaStream_t s) {
    if (mode == 0) k_fm_gather<NST, 0><<<B.n, kFmThreads, 0, s>>>(B, W, rows, A, M, NS, g, fd);
    else k_fm_gather<NST, 1><<<B.n, kFmThreads, 0, s>>>(B, W, rows, A, M, NS, g, fd);
}

}  // namespace

extern "C" {

const char* xi_fm_last_error(void) { return g_err; }

int xi_fm_scatter(const XiFmBoxes* boxes, const XiFmWindow* win, const float* I, const float* beta, float* mu,
                  void* stream) {
    int rc = check_boxes(boxes, win);
    if (rc) return rc;
    if (boxes->n == 0) return XI_OK;
    if (!I || !mu) return fm_fail(XI_E_ARG, "xi_fm_scatter: null I or mu");
    k_fm_scatter<<<boxes->n, kFmThreads, 0, (cudaStream_t)stream>>>(*boxes, *win, I, beta, mu);
    return launch_check("xi_fm_scatter");
}

int xi_fm_gather(const XiFmBoxes* boxes, const XiFmWindow* win, const int64_t* rows, const float* A, const float* M,
                 const void* NS, int ns_type, int mode, float* g, float* fd, void* stream) {
    int rc = check_boxes(boxes, win);
    if (rc) return rc;
    if (boxes->n == 0) return XI_OK;
    if (!M || !NS || !g) return fm_fail(XI_E_ARG, "xi_fm_gather: null M, NS or g");
    if (mode == 0 && !A) return fm_fail(XI_E_ARG, "xi_fm_gather: mode 0 needs A");
    if (mode == 1 && !fd) return fm_fail(XI_E_ARG, "xi_fm_gather: mode 1 needs fd");
    if (mode != 0 && mode != 1) return fm_fail(XI_E_ARG, "xi_fm_gather: mode 0 or 1");
    cudaStream_t s = (cudaStream_t)stream;
    switch (ns_type) {
        case XI_FM_NS_I16: launch_gather<int16_t>(*boxes, *win, rows, A, M, NS, mode, g, fd, s); break;
        case XI_FM_NS_I32: launch_gather<int32_t>(*boxes, *win, rows, A, M, NS, mode, g, fd, s); break;
        case XI_FM_NS_F32: launch_gather<float>(*boxes, *win, rows, A, M, NS, mode, g, fd, s); break;
        default: return fm_fail(XI_E_ARG, "xi_fm_gather: ns_type");
    }
    return launch_check("xi_fm_gather");
}

}  // extern "C"
