// k_fragile.cu -- exact correlations of the surviving candidates with the
// fragile windows of a length.
//
// No counterpart in the reference, whose FP32 refine (gpu_global_discords_refine,
// src/PD3_kernels.cuh:582-662) evaluates every pair the same way.  Here the
// refine kernels evaluate a pair (candidate c, window j) with an error bound
// g_j that grows with |x_j - s| / |x_j - mu_j| for the shift s of j's tile
// (window_bound in paddi_internal.cuh).  Windows whose bound exceeds the
// guard band -- near-flat windows far from their tile's level, series with a
// large offset and small local variance -- are "fragile": the refine uses
// their correlations only lowered by their own bound (to prune) and keeps no
// upper estimate of them, and this kernel, run after the refine's last round,
// evaluates them in FP64 against every candidate still unpruned:
//     rho = sum_k (x_c+k - mu_c)(x_f+k - mu_f) inv_c inv_f,
// both windows centred on their own FP64 means, so the error is ~1e-14 of
// the result whatever the offset.  A correlation above thr + 1e-7 prunes the
// candidate (the margin covers the FP32 rounding of thr); every value enters
// the candidate's kept maximum.
//
// Work items: (8 candidates of the list, 256 fragile windows); one thread per
// fragile window reads its window once for all 8 candidates (8 loads in
// flight at a time), whose centred values sit in shared memory.  Fragile windows come in runs (tile prep and
// the FP32 scan append them in index order within each warp), so the series
// reads of a warp are mostly contiguous.
#include <float.h>

#include "paddi_internal.cuh"

using paddi::f2ord;

namespace {

constexpr int FG_THREADS = 256;
constexpr int FG_CAND = 8;     // candidates per work item
constexpr int FG_UNROLL = 8;   // series loads in flight per thread
constexpr int FG_MAXM = 1024;

__global__ void __launch_bounds__(FG_THREADS)
k_fragile(const float *__restrict__ x, const double *__restrict__ mu64,
          const double *__restrict__ inv64, const int32_t *__restrict__ cand,
          const int32_t *__restrict__ list, const int32_t *__restrict__ list_count,
          uint8_t *pruned, uint32_t *rho_max, const int32_t *__restrict__ frag,
          const int32_t *__restrict__ frag_count, int32_t m, float thr, int32_t col_lo,
          int32_t col_hi)
{
    extern __shared__ __align__(16) double fg_a[]; // [FG_CAND][mpad]: centred candidates
    __shared__ int cw[FG_CAND], cp[FG_CAND], live[FG_CAND];
    __shared__ int s_any;
    __shared__ double red[FG_CAND][FG_THREADS / 32];
    const int C = *list_count, F = *frag_count;
    if (C <= 0 || F <= 0) return;
    const int mpad = (m + FG_UNROLL - 1) / FG_UNROLL * FG_UNROLL;
    const int groups = (C + FG_CAND - 1) / FG_CAND;
    const int chunks = (F + FG_THREADS - 1) / FG_THREADS;
    const long long total = (long long)groups * chunks;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (long long item = blockIdx.x; item < total; item += gridDim.x) {
        const int grp = (int)(item % groups), chunk = (int)(item / groups);
        __syncthreads();
        if (t == 0) s_any = 0;
        __syncthreads();
        if (t < FG_CAND) {
            const int li = grp * FG_CAND + t;
            const int pos = li < C ? list[li] : -1;
            cp[t] = pos;
            cw[t] = pos >= 0 ? cand[pos] : 0;
            live[t] = pos >= 0 && !__ldcg(pruned + pos);
            if (live[t]) s_any = 1;
        }
        __syncthreads();
        if (!s_any) continue;
        for (int e = t; e < FG_CAND * mpad; e += FG_THREADS) {
            const int c = e / mpad, k = e - c * mpad;
            fg_a[e] = (live[c] && k < m) ? (double)x[cw[c] + k] - mu64[cw[c]] : 0.0;
        }
        __syncthreads();
        double best[FG_CAND];
#pragma unroll
        for (int c = 0; c < FG_CAND; ++c) best[c] = -INFINITY;
        const int fi = chunk * FG_THREADS + t;
        const int f = fi < F ? frag[fi] : -1;
        if (f >= col_lo && f < col_hi) {
            const double mf = mu64[f], ivf = inv64[f];
            double acc[FG_CAND];
#pragma unroll
            for (int c = 0; c < FG_CAND; ++c) acc[c] = 0.0;
            for (int k0 = 0; k0 < mpad; k0 += FG_UNROLL) {
                float v[FG_UNROLL]; // independent loads first, then the FMAs
#pragma unroll
                for (int u = 0; u < FG_UNROLL; ++u) v[u] = k0 + u < m ? __ldg(x + f + k0 + u) : 0.f;
#pragma unroll
                for (int u = 0; u < FG_UNROLL; ++u) {
                    const double y = k0 + u < m ? (double)v[u] - mf : 0.0;
#pragma unroll
                    for (int c = 0; c < FG_CAND; ++c)
                        acc[c] = fma(fg_a[c * mpad + k0 + u], y, acc[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < FG_CAND; ++c) {
                const int d = cw[c] > f ? cw[c] - f : f - cw[c];
                if (live[c] && d >= m - 1) best[c] = acc[c] * inv64[cw[c]] * ivf;
            }
        }
#pragma unroll
        for (int c = 0; c < FG_CAND; ++c) {
            double v = best[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            if (lane == 0) red[c][warp] = v;
        }
        __syncthreads();
        if (t < FG_CAND && live[t]) {
            double v = -INFINITY;
            for (int w = 0; w < FG_THREADS / 32; ++w) v = fmax(v, red[t][w]);
            if (v > -INFINITY) {
                atomicMax(rho_max + cp[t], f2ord((float)v));
                if (v > (double)thr + 1e-7) pruned[cp[t]] = 1;
            }
        }
    }
}

} // namespace

cudaError_t paddi_launch_fragile(const float *x, const double *mu64, const double *inv64,
                                 const int32_t *cand, const int32_t *list,
                                 const int32_t *list_count, uint8_t *pruned, uint32_t *rho_max,
                                 const int32_t *frag, const int32_t *frag_count, int32_t m,
                                 float thr, int32_t col_lo, int32_t col_hi, int32_t num_sms,
                                 cudaStream_t st)
{
    if (m > FG_MAXM) return cudaErrorInvalidValue;
    const int mpad = (m + FG_UNROLL - 1) / FG_UNROLL * FG_UNROLL;
    const size_t smem = sizeof(double) * (size_t)FG_CAND * mpad;
    cudaError_t e = paddi_raise_smem_limit((const void *)k_fragile, smem);
    if (e != cudaSuccess) return e;
    k_fragile<<<num_sms * 2, FG_THREADS, smem, st>>>(x, mu64, inv64, cand, list, list_count,
                                                    pruned, rho_max, frag, frag_count, m, thr,
                                                    col_lo, col_hi);
    return cudaGetLastError();
}
