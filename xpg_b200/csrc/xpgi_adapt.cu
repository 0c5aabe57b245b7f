// Per-block adaptation of the rocking curve on the device (include/xpgi.h, "Adaptation"): the sigma_M grid search
// and the normal equations of the rocking-curve mixture fit. XPG evaluates both in numpy on the host from the
// block's strong reflections (xpg/integrate.py:404-461, :1130-1154); here one thread evaluates one reflection's
// frames, float64 throughout, and every reduction runs in a fixed order (the results do not depend on the launch).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "xpgi.h"
#include "xpgi_internal.h"

namespace {

constexpr int kFrames = 65;          // fz columns (the deepest box)
constexpr int kK = XI_RC_K;          // mixture components
constexpr int kNT = 256;
constexpr int kGramEntries = kK * (kK + 1) / 2 + kK;   // upper triangle of A^T A, then A^T y
constexpr int kGramBlocks = 148;
constexpr int kTile = 128;           // (reflection, frame) pairs per shared-memory tile of the Gram kernel

// numpy's pairwise sum of a 65-element row: eight running sums over the first 64 values, combined as
// ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7)), then the last value
__device__ __forceinline__ double row_sum65(const double* a) {
    double r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    for (int i = 8; i < 64; i += 8) {
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    }
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    return res + a[64];
}

__device__ __forceinline__ double z_to_phi(const XiRocking& q, double z) { return q.phi0 + q.osc * (z - q.z_shift); }

__device__ __forceinline__ double rc_centre(int k) { return k == kK - 1 ? 3.5 : (double)k * 0.35 + (-3.5); }

template <int NT>
__device__ double block_sum1(double v, double* scratch) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; ++w) s += scratch[w];
    return s;
}

// cost of grid width grid[blockIdx.x] (deg): sum over rows with a positive total of tot * (frac - R)^2
__global__ void __launch_bounds__(kNT) k_rock_costs(XiRocking q, const double* __restrict__ grid,
                                                    double* __restrict__ cost) {
    __shared__ double scratch[kNT / 32];
    const double sm = grid[blockIdx.x];
    const double sq2 = sqrt(2.0);
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < q.n; i += kNT) {
        const double* f = q.fz + (size_t)i * kFrames;
        const double tot = row_sum65(f);
        if (!(tot > 0.0)) continue;
        const double phi = q.phi[i];
        const double s = sm / fabs(q.zeta[i]) * sq2;
        double R[kFrames];
        for (int z = 0; z < kFrames; ++z) {
            const double k = (double)q.iz0[i] + (double)z;
            const double a = z_to_phi(q, k), b = z_to_phi(q, k + 1.0);
            const double lo = fmin(a, b), hi = fmax(a, b);
            R[z] = 0.5 * (erf((hi - phi) / s) - erf((lo - phi) / s));
        }
        const double rs = fmax(row_sum65(R), 1e-9);
        double c = 0.0;
        for (int z = 0; z < kFrames; ++z) {
            const double d = f[z] / tot - R[z] / rs;
            c += tot * (d * d);
        }
        acc += c;
    }
    const double s = block_sum1<kNT>(acc, scratch);
    if (threadIdx.x == 0) cost[blockIdx.x] = s;
}

__global__ void k_rock_tot(XiRocking q, double* __restrict__ tot) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < q.n) tot[i] = fmax(row_sum65(q.fz + (size_t)i * kFrames), 1e-9);
}

// partial A^T A / A^T y of one contiguous range of (reflection, frame) pairs; A = B sqrt(tot), y = fz / tot sqrt(tot)
// with B the frame integrals of the 21 mixture components at width sm (rad), centred on the predicted angle
__global__ void __launch_bounds__(kNT) k_rock_gram(XiRocking q, double sm, const double* __restrict__ tot,
                                                   int64_t per_block, double* __restrict__ part) {
    __shared__ double At[kTile][kK + 1];
    const int64_t n_pairs = q.n * kFrames;
    const int64_t b0 = (int64_t)blockIdx.x * per_block;
    const int64_t b1 = b0 + per_block < n_pairs ? b0 + per_block : n_pairs;
    const int t = threadIdx.x;
    int ek = 0, el = 0;                          // this thread's entry: (k, l) with k <= l, or the rhs row k
    if (t < kGramEntries) {
        if (t < kK * (kK + 1) / 2) {
            int r = t, k = 0;
            while (r >= kK - k) {
                r -= kK - k;
                ++k;
            }
            ek = k;
            el = k + r;
        } else {
            ek = t - kK * (kK + 1) / 2;
            el = kK;                             // the y column
        }
    }
    const double sq2 = sqrt(2.0), rad = M_PI / 180.0;
    double acc = 0.0;
    for (int64_t p0 = b0; p0 < b1; p0 += kTile) {
        if (t < kTile) {
            const int64_t p = p0 + t;
            if (p < b1) {
                const int64_t i = p / kFrames;
                const int z = (int)(p - i * kFrames);
                const double st = sqrt(tot[i]);
                const double k = (double)q.iz0[i] + (double)z;
                const double a = z_to_phi(q, k), b = z_to_phi(q, k + 1.0);
                const double lo = fmin(a, b) * rad, hi = fmax(a, b) * rad;
                const double pc = q.phi[i] * rad;
                const double s = sm / fmax(fabs(q.zeta[i]), 1e-3);
                const double sw = s * 0.25 * sq2;
                for (int c = 0; c < kK; ++c) {
                    const double cs = rc_centre(c) * s;
                    const double ea = (hi - pc - cs) / sw, eb = (lo - pc - cs) / sw;
                    At[t][c] = (0.5 * (erf(ea) - erf(eb))) * st;
                }
                At[t][kK] = q.fz[(size_t)i * kFrames + z] / tot[i] * st;
            } else {
                for (int c = 0; c <= kK; ++c) At[t][c] = 0.0;
            }
        }
        __syncthreads();
        if (t < kGramEntries) {
            const int m = (int)(b1 - p0 < kTile ? b1 - p0 : kTile);
            for (int j = 0; j < m; ++j) acc += At[j][ek] * At[j][el];
        }
        __syncthreads();
    }
    if (t < kGramEntries) part[(size_t)blockIdx.x * kGramEntries + t] = acc;
}

__global__ void k_rock_gram_sum(const double* __restrict__ part, int nb, double* __restrict__ gram,
                                double* __restrict__ rhs) {
    const int t = threadIdx.x;
    if (t >= kGramEntries) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[(size_t)b * kGramEntries + t];
    if (t < kK * (kK + 1) / 2) {
        int r = t, k = 0;
        while (r >= kK - k) {
            r -= kK - k;
            ++k;
        }
        const int l = k + r;
        gram[k * kK + l] = s;
        gram[l * kK + k] = s;
    } else {
        rhs[t - kK * (kK + 1) / 2] = s;
    }
}

int rocking_check(const XiRocking* q) {
    if (!q) return xi_fail(XI_E_ARG, "rocking: null argument");
    if (q->n < 0) return xi_fail(XI_E_ARG, "rocking: negative size");
    if (q->n && (!q->fz || !q->iz0 || !q->phi || !q->zeta)) return xi_fail(XI_E_ARG, "rocking: null column");
    if (q->n > ((int64_t)1 << 40) / kFrames) return xi_fail(XI_E_LIMIT, "rocking: too many rows");
    return XI_OK;
}

}  // namespace

extern "C" {

int xi_rocking_costs(const XiRocking* q, const double* grid, int n_grid, double* cost, void* stream) {
    int rc = rocking_check(q);
    if (rc) return rc;
    if (n_grid < 0 || (n_grid && (!grid || !cost))) return xi_fail(XI_E_ARG, "xi_rocking_costs: grid");
    if (n_grid == 0) return XI_OK;
    k_rock_costs<<<n_grid, kNT, 0, (cudaStream_t)stream>>>(*q, grid, cost);
    return xi_cuda_check("xi_rocking_costs");
}

size_t xi_rocking_gram_workspace(const XiRocking* q) {
    if (!q || q->n < 0) return 0;
    return (((size_t)q->n * sizeof(double) + 255) / 256 * 256) + (size_t)kGramBlocks * kGramEntries * sizeof(double);
}

int xi_rocking_gram(const XiRocking* q, double sm, void* ws, size_t ws_bytes, double* gram, double* rhs,
                    void* stream) {
    int rc = rocking_check(q);
    if (rc) return rc;
    if (!gram || !rhs) return xi_fail(XI_E_ARG, "xi_rocking_gram: null output");
    if (!ws || ws_bytes < xi_rocking_gram_workspace(q)) return xi_fail(XI_E_ARG, "xi_rocking_gram: workspace");
    cudaStream_t s = (cudaStream_t)stream;
    double* tot = static_cast<double*>(ws);
    double* part = reinterpret_cast<double*>(static_cast<char*>(ws) + ((size_t)q->n * sizeof(double) + 255) / 256 * 256);
    const int64_t n_pairs = q->n * kFrames;
    int64_t per_block = (n_pairs + kGramBlocks - 1) / kGramBlocks;
    per_block = (per_block + kTile - 1) / kTile * kTile;
    const int nb = n_pairs ? (int)((n_pairs + per_block - 1) / per_block) : 0;
    if (q->n) k_rock_tot<<<(unsigned)((q->n + 255) / 256), 256, 0, s>>>(*q, tot);
    if (nb) k_rock_gram<<<nb, kNT, 0, s>>>(*q, sm, tot, per_block, part);
    k_rock_gram_sum<<<1, kNT, 0, s>>>(part, nb, gram, rhs);
    return xi_cuda_check("xi_rocking_gram");
}

}  // extern "C"
