// k_fragile.cu -- exact correlations of the surviving candidates with the
// fragile windows of a length.
//
// No counterpart in the reference, whose FP32 refine (gpu_global_discords_refine,
// src/PD3_kernels.cuh:582-662) evaluates every pair the same way.  Here the
// refine kernels evaluate a pair (candidate c, window j) with an error bound
// g_j that grows with |x_j - s| / |x_j - mu_j| for the shift s of j's tile
// (window_bound in paddi_internal.cuh).  Windows whose bound exceeds the
// guard band -- near-flat windows far from their tile's level, series with a
// large offset and small local variance -- are "fragile": the tensor-core
// refine skips them (the FP32 refine uses them lowered by their own bound, to
// prune), and this kernel, run after the refine's last round, evaluates them
// in FP64 against every candidate still unpruned:
//     rho = sum_k (x_c+k - mu_c)(x_f+k - mu_f) inv_c inv_f,
// both windows centred on their own FP64 means, so the error is ~1e-14 of
// the result whatever the offset.  A correlation above thr + 1e-7 prunes the
// candidate (the margin covers the FP32 rounding of thr); every value enters
// the candidate's kept maximum.
//
// Work items: (a group of 8 entries of the candidate list, 256 consecutive
// entries of the fragile list).  The group's centred candidate values sit in
// shared memory (read as broadcasts, two terms per load); each thread owns
// one fragile window, reads its values once per 4-candidate half of the group
// straight from the series (consecutive addresses per thread, so 7 of 8
// loads hit L1) and keeps 4 FP64 accumulators.  Halves whose candidates are
// all pruned, and items with no live candidate, are skipped.
#include <float.h>

#include "paddi_internal.cuh"

using paddi::f2ord;

namespace {

constexpr int FG_THREADS = 256; // fragile windows per item (one per thread)
constexpr int FG_CAND = 8;      // candidate-list entries per item
constexpr int FG_HALF = 4;      // accumulators per thread
constexpr int FG_MAXM = 1024;

__global__ void __launch_bounds__(FG_THREADS)
k_fragile(const float *__restrict__ x, const double *__restrict__ mu64,
          const double *__restrict__ inv64, const int32_t *__restrict__ cand,
          const int32_t *__restrict__ list, const int32_t *__restrict__ list_count,
          uint8_t *pruned, uint32_t *rho_max, const int32_t *__restrict__ frag,
          const int32_t *__restrict__ frag_count, int32_t m, float thr, int32_t col_lo,
          int32_t col_hi)
{
    // [FG_CAND][mp] centred candidate values, mp = m rounded up to even
    extern __shared__ __align__(16) double fg_a[];
    __shared__ int cw[FG_CAND], cp[FG_CAND], live[FG_CAND];
    __shared__ double civ[FG_CAND];
    __shared__ double best_s[FG_CAND][FG_THREADS / 32];
    __shared__ int s_any;
    const int C = *list_count, F = *frag_count;
    if (C <= 0 || F <= 0) return;
    const int mp = (m + 1) & ~1;
    const int groups = (C + FG_CAND - 1) / FG_CAND;
    const int chunks = (F + FG_THREADS - 1) / FG_THREADS;
    const long long total = (long long)groups * chunks;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (long long item = blockIdx.x; item < total; item += gridDim.x) {
        const int grp = (int)(item % groups), chunk = (int)(item / groups);
        __syncthreads(); // the previous item's shared data is consumed
        if (t == 0) s_any = 0;
        __syncthreads();
        if (t < FG_CAND) {
            const int li = grp * FG_CAND + t;
            const int pos = li < C ? list[li] : -1;
            const int w = pos >= 0 ? cand[pos] : 0;
            cp[t] = pos;
            cw[t] = w;
            live[t] = pos >= 0 && !__ldcg(pruned + pos);
            civ[t] = inv64[w];
            if (live[t]) atomicOr(&s_any, 1);
        }
        __syncthreads();
        if (!s_any) continue;
        for (int e = t; e < FG_CAND * mp; e += FG_THREADS) {
            const int c = e / mp, k = e - c * mp;
            fg_a[e] = (live[c] && k < m) ? (double)x[cw[c] + k] - mu64[cw[c]] : 0.0;
        }
        __syncthreads();
        const int fi = chunk * FG_THREADS + t;
        const int f = fi < F ? frag[fi] : -1;
        const bool fok = f >= col_lo && f < col_hi;
        double b[FG_CAND];
#pragma unroll
        for (int c = 0; c < FG_CAND; ++c) b[c] = -INFINITY;
#pragma unroll
        for (int h = 0; h < FG_CAND / FG_HALF; ++h) {
            const int c0 = h * FG_HALF;
            bool any = false;
#pragma unroll
            for (int c = 0; c < FG_HALF; ++c) any |= live[c0 + c] != 0;
            if (!any || !fok) continue; // any: uniform over the block
            const double mf = mu64[f];
            const float *y = x + f;
            const double2 *a2 = reinterpret_cast<const double2 *>(fg_a + c0 * mp);
            const int mh = mp >> 1;
            double acc[FG_HALF];
#pragma unroll
            for (int c = 0; c < FG_HALF; ++c) acc[c] = 0.0;
#pragma unroll 4
            for (int q = 0; q < mh; ++q) {
                // terms 2q, 2q+1 (the even padding term has zero candidate values)
                const double v0 = (double)__ldg(y + 2 * q) - mf;
                const double v1 = 2 * q + 1 < m ? (double)__ldg(y + 2 * q + 1) - mf : 0.0;
#pragma unroll
                for (int c = 0; c < FG_HALF; ++c) {
                    const double2 av = a2[c * mh + q];
                    acc[c] = fma(av.y, v1, fma(av.x, v0, acc[c]));
                }
            }
            const double ivf = inv64[f];
#pragma unroll
            for (int c = 0; c < FG_HALF; ++c) {
                const int ci = c0 + c;
                const int d = cw[ci] > f ? cw[ci] - f : f - cw[ci];
                if (live[ci] && d >= m - 1) b[ci] = acc[c] * civ[ci] * ivf;
            }
        }
        // maxima over the item's windows, per candidate
#pragma unroll
        for (int c = 0; c < FG_CAND; ++c) {
            double v = b[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            if (lane == 0) best_s[c][warp] = v;
        }
        __syncthreads();
        if (t < FG_CAND && live[t]) {
            double v = -INFINITY;
#pragma unroll
            for (int q = 0; q < FG_THREADS / 32; ++q) v = fmax(v, best_s[t][q]);
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
    if (m > FG_MAXM || m < 3) return cudaErrorInvalidValue;
    const size_t smem = sizeof(double) * (size_t)FG_CAND * (size_t)((m + 1) & ~1);
    cudaError_t e = paddi_raise_smem_limit((const void *)k_fragile, smem);
    if (e != cudaSuccess) return e;
    k_fragile<<<num_sms * 4, FG_THREADS, smem, st>>>(x, mu64, inv64, cand, list, list_count,
                                                    pruned, rho_max, frag, frag_count, m, thr,
                                                    col_lo, col_hi);
    return cudaGetLastError();
}
