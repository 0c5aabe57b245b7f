// Device side of the frames' transfer encoding (include/xpgi.h, "Transfer encoding"), the bit unshuffle of
// bitshuffle-LZ4 frames, and xi_upload (small uploads read by a kernel from mapped page-locked host memory).
// The unpacking: one byte per pixel widened to
// uint32, then the exception pairs written over the escaped pixels. A CTA widens a span of kSpan pixels with 16-byte
// loads and stores, then writes the exceptions inside its span (found by a binary search of the sorted indices), so
// every pixel is written by one CTA, the exceptions after the byte codes.
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpgi.h"
#include "xpgi_internal.h"

namespace {

constexpr int kNT = 256;
constexpr int64_t kSpan = (int64_t)kNT * 16 * 4;   // pixels per CTA: four 16-byte plane loads per thread

__device__ __forceinline__ uint32_t widen(uint32_t b) { return b == XI_PACK_FLAGGED ? 0xFFFFFFFFu : b; }

// One span (kSpan pixels, index `span`) of a packed run widened into out: the byte codes, then the span's
// exception pairs.
__device__ __forceinline__ void unpack_span(const uint8_t* __restrict__ plane, int64_t n,
                                            const uint32_t* __restrict__ exc, int64_t n_exc,
                                            uint32_t* __restrict__ out, int64_t span) {
    const int64_t a = span * kSpan;
    const int64_t b = a + kSpan < n ? a + kSpan : n;
    for (int64_t p = a + (int64_t)threadIdx.x * 16; p < b; p += (int64_t)kNT * 16) {
        if (p + 16 <= b) {
            const uint4 v = *reinterpret_cast<const uint4*>(plane + p);
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
            uint4* o = reinterpret_cast<uint4*>(out + p);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                o[q] = make_uint4(widen(w[q] & 0xFFu), widen((w[q] >> 8) & 0xFFu), widen((w[q] >> 16) & 0xFFu),
                                  widen(w[q] >> 24));
        } else {
            for (int64_t i = p; i < b; ++i) out[i] = widen(plane[i]);
        }
    }
    if (n_exc == 0) return;
    __syncthreads();                         // the byte codes of the span are written before the exceptions
    __shared__ int64_t s_lo;
    if (threadIdx.x == 0) {                  // first exception with index >= a
        int64_t lo = 0, hi = n_exc;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((int64_t)exc[2 * mid] < a) lo = mid + 1;
            else hi = mid;
        }
        s_lo = lo;
    }
    __syncthreads();
    for (int64_t k = s_lo + threadIdx.x; k < n_exc; k += kNT) {
        const int64_t i = exc[2 * k];
        if (i >= b) break;
        out[i] = exc[2 * k + 1];
    }
}

__global__ void __launch_bounds__(kNT) k_unpack_u8(const uint8_t* __restrict__ plane, int64_t n,
                                                   const uint32_t* __restrict__ exc, int64_t n_exc,
                                                   uint32_t* __restrict__ out) {
    unpack_span(plane, n, exc, n_exc, out, blockIdx.x);
}

// Several packed frames at once (blockIdx.y: the frame); a raw frame's plane holds its uint32 values (copied).
__global__ void __launch_bounds__(kNT) k_unpack_u8_frames(const XiPackedFrame* __restrict__ fr, int64_t n,
                                                          uint32_t* __restrict__ out, int64_t stride) {
    const XiPackedFrame f = fr[blockIdx.y];
    uint32_t* o = out + (int64_t)blockIdx.y * stride;
    if (f.raw) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(f.plane);
        const int64_t a = (int64_t)blockIdx.x * kSpan;
        const int64_t b = a + kSpan < n ? a + kSpan : n;
        for (int64_t p = a + threadIdx.x; p < b; p += kNT) o[p] = src[p];
        return;
    }
    unpack_span(f.plane, n, f.exc, f.n_exc, o, blockIdx.x);
}

// byte copy from mapped host memory; the 16-byte body when both ends are 16-byte aligned, bytes otherwise
__global__ void __launch_bounds__(kNT) k_upload(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                                int64_t bytes, int vec) {
    const int64_t stride = (int64_t)gridDim.x * kNT;
    const int64_t t0 = (int64_t)blockIdx.x * kNT + threadIdx.x;
    int64_t done = 0;
    if (vec) {
        const int64_t n16 = bytes >> 4;
        for (int64_t i = t0; i < n16; i += stride)
            reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
        done = n16 << 4;
    }
    for (int64_t i = done + t0; i < bytes; i += stride) dst[i] = src[i];
}

// 8 x 8 bit-matrix transpose of a 64-bit word (bit 8 r + c <-> bit 8 c + r) by three delta swaps (the standard
// method, Hacker's Delight 7-3)
__device__ __forceinline__ unsigned long long transpose8(unsigned long long x) {
    unsigned long long t;
    t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
    x = x ^ t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
    x = x ^ t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
    x = x ^ t ^ (t << 28);
    return x;
}

// One thread per group of 8 elements. In a block of m8 = belem / 8 groups, bit plane 8 b + k (bit k of byte b of
// every element) is a row of m8 bytes, element 8 g + j at bit j of the row's byte g: the thread reads byte g of the
// 8 rows of byte b (consecutive threads, consecutive bytes), transposes them into byte b of its 8 elements. The
// frame's last partial block is shuffled as one block of its multiple-of-8 elements; its n % 8 elements are stored
// as they are (the last thread copies them). uint16 elements are widened, the all-ones value to 0xFFFFFFFF.
template <int E>
__global__ void __launch_bounds__(kNT) k_bitunshuffle(const uint8_t* __restrict__ in, int64_t n, int64_t belem,
                                                      uint32_t* __restrict__ out, int vec) {
    const int64_t n8 = n / 8;
    const int64_t G = (int64_t)blockIdx.x * kNT + threadIdx.x;
    const int64_t nf = n / belem;                              // full blocks
    if (G < n8) {
        const int64_t full_groups = nf * (belem / 8);
        int64_t base, g, m8;
        if (G < full_groups) {
            const int64_t k = G / (belem / 8);
            g = G - k * (belem / 8);
            m8 = belem / 8;
            base = k * belem * E;
        } else {
            g = G - full_groups;
            m8 = (n - nf * belem) / 8;
            base = nf * belem * E;
        }
        uint32_t v[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
#pragma unroll
        for (int b = 0; b < E; ++b) {
            unsigned long long x = 0ull;
#pragma unroll
            for (int k = 0; k < 8; ++k) x |= (unsigned long long)in[base + (int64_t)(8 * b + k) * m8 + g] << (8 * k);
            x = transpose8(x);
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] |= (uint32_t)((x >> (8 * j)) & 0xFFull) << (8 * b);
        }
        if (E == 2) {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = v[j] == 0xFFFFu ? 0xFFFFFFFFu : v[j];
        }
        if (vec) {                                             // out 16-byte aligned: two 16-byte stores
            uint4* o = reinterpret_cast<uint4*>(out + 8 * G);
            o[0] = make_uint4(v[0], v[1], v[2], v[3]);
            o[1] = make_uint4(v[4], v[5], v[6], v[7]);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) out[8 * G + j] = v[j];
        }
    } else if (G == n8) {
        for (int64_t i = 8 * n8; i < n; ++i) {                  // the trailing n % 8 elements, stored as they are
            uint32_t e = 0u;
            for (int b = 0; b < E; ++b) e |= (uint32_t)in[i * E + b] << (8 * b);
            out[i] = (E == 2 && e == 0xFFFFu) ? 0xFFFFFFFFu : e;
        }
    }
}

}  // namespace

extern "C" int xi_bitunshuffle(const uint8_t* in, int64_t n_elem, int esize, int64_t block_elems, uint32_t* out,
                               void* stream) {
    if (n_elem < 0 || (n_elem && (!in || !out))) return xi_fail(XI_E_ARG, "xi_bitunshuffle: null pointer or negative size");
    if (esize != 2 && esize != 4) return xi_fail(XI_E_ARG, "xi_bitunshuffle: element size must be 2 or 4");
    if (block_elems <= 0 || block_elems % 8) return xi_fail(XI_E_ARG, "xi_bitunshuffle: block not a multiple of 8");
    if ((uintptr_t)out & 3) return xi_fail(XI_E_ARG, "xi_bitunshuffle: out must be 4-byte aligned");
    const int vec = ((uintptr_t)out & 15) == 0;
    if (n_elem == 0) return XI_OK;
    const int64_t threads = n_elem / 8 + 1;
    const unsigned grid = (unsigned)((threads + kNT - 1) / kNT);
    if (esize == 4) k_bitunshuffle<4><<<grid, kNT, 0, (cudaStream_t)stream>>>(in, n_elem, block_elems, out, vec);
    else k_bitunshuffle<2><<<grid, kNT, 0, (cudaStream_t)stream>>>(in, n_elem, block_elems, out, vec);
    return xi_cuda_check("xi_bitunshuffle");
}

extern "C" int xi_upload(const void* src, void* dst, int64_t bytes, void* stream) {
    if (bytes < 0 || (bytes && (!src || !dst))) return xi_fail(XI_E_ARG, "xi_upload: null pointer or negative size");
    if (bytes == 0) return XI_OK;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, src) != cudaSuccess) {
        cudaGetLastError();
        return xi_fail(XI_E_ARG, "xi_upload: src is not page-locked host memory");
    }
    if (at.type != cudaMemoryTypeHost || !at.devicePointer)
        return xi_fail(XI_E_ARG, "xi_upload: src is not mapped page-locked host memory");
    const uint8_t* s = static_cast<const uint8_t*>(at.devicePointer);
    const int vec = !((uintptr_t)s & 15) && !((uintptr_t)dst & 15);
    int64_t grid = (bytes / (vec ? 16 : 1) + kNT - 1) / kNT;
    grid = grid < 1 ? 1 : (grid > 1184 ? 1184 : grid);          // 8 CTAs per SM at most
    k_upload<<<(unsigned)grid, kNT, 0, (cudaStream_t)stream>>>(s, static_cast<uint8_t*>(dst), bytes, vec);
    return xi_cuda_check("xi_upload");
}

extern "C" int xi_unpack_u8_frames(const XiPackedFrame* frames, int n_frames, int64_t n, uint32_t* out, int64_t stride,
                                   void* stream) {
    if (n < 0 || n_frames < 0 || stride < n || (n && n_frames && (!frames || !out)))
        return xi_fail(XI_E_ARG, "xi_unpack_u8_frames: null pointer or bad size");
    if (n > XI_PACK_MAX_PIXELS || n_frames > 65535) return xi_fail(XI_E_LIMIT, "xi_unpack_u8_frames: too large");
    if (((uintptr_t)out & 15) || (stride & 3)) return xi_fail(XI_E_ARG, "xi_unpack_u8_frames: out / stride alignment");
    if (n == 0 || n_frames == 0) return XI_OK;
    const dim3 grid((unsigned)((n + kSpan - 1) / kSpan), (unsigned)n_frames);
    k_unpack_u8_frames<<<grid, kNT, 0, (cudaStream_t)stream>>>(frames, n, out, stride);
    return xi_cuda_check("xi_unpack_u8_frames");
}

extern "C" int xi_unpack_u8(const uint8_t* plane, int64_t n, const uint32_t* exc, int64_t n_exc, uint32_t* out,
                            void* stream) {
    if (n < 0 || n_exc < 0 || (n && (!plane || !out)) || (n_exc && !exc))
        return xi_fail(XI_E_ARG, "xi_unpack_u8: null pointer or negative size");
    if (n > XI_PACK_MAX_PIXELS) return xi_fail(XI_E_LIMIT, "xi_unpack_u8: more than XI_PACK_MAX_PIXELS pixels");
    if (((uintptr_t)plane & 15) || ((uintptr_t)out & 15) || ((uintptr_t)exc & 3))
        return xi_fail(XI_E_ARG, "xi_unpack_u8: plane and out must be 16-byte aligned");
    if (n == 0) return XI_OK;
    const int64_t grid = (n + kSpan - 1) / kSpan;
    k_unpack_u8<<<(unsigned)grid, kNT, 0, (cudaStream_t)stream>>>(plane, n, exc, n_exc, out);
    return xi_cuda_check("xi_unpack_u8");
}
