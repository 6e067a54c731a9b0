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
// Work items: (8 candidates of the list, 64 consecutive entries of the
// fragile list).  Fragile windows come in runs (tile prep and the FP32 scan
// append them in index order within each warp), so an item's windows usually
// span a short stretch of the series: it is staged in shared memory once and
// each thread evaluates one window against 2 of the 8 candidates (whose
// centred values also sit in shared memory).  An item whose windows span more
// than FG_SPAN values reads the series from global memory instead.
#include <float.h>
#include <limits.h>

#include "paddi_internal.cuh"

using paddi::f2ord;

namespace {

constexpr int FG_THREADS = 256;
constexpr int FG_CAND = 8;     // candidates per work item
constexpr int FG_WIN = 64;     // fragile windows per work item
constexpr int FG_SPAN = 3072;  // longest staged stretch of the series
constexpr int FG_MAXM = 1024;
static_assert(FG_THREADS == FG_WIN * FG_CAND / 2, "one window and two candidates per thread");

__global__ void __launch_bounds__(FG_THREADS)
k_fragile(const float *__restrict__ x, const double *__restrict__ mu64,
          const double *__restrict__ inv64, const int32_t *__restrict__ cand,
          const int32_t *__restrict__ list, const int32_t *__restrict__ list_count,
          uint8_t *pruned, uint32_t *rho_max, const int32_t *__restrict__ frag,
          const int32_t *__restrict__ frag_count, int32_t m, float thr, int32_t col_lo,
          int32_t col_hi)
{
    extern __shared__ __align__(16) double fg_a[]; // [FG_CAND][m]: centred candidates
    __shared__ float xs[FG_SPAN];                  // the item's stretch of the series
    __shared__ int cw[FG_CAND], cp[FG_CAND], live[FG_CAND];
    __shared__ int fw[FG_WIN];
    __shared__ double best_s[FG_CAND][FG_THREADS / 32];
    __shared__ int s_any, s_lo, s_hi;
    const int C = *list_count, F = *frag_count;
    if (C <= 0 || F <= 0) return;
    const int groups = (C + FG_CAND - 1) / FG_CAND;
    const int chunks = (F + FG_WIN - 1) / FG_WIN;
    const long long total = (long long)groups * chunks;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wi = t & (FG_WIN - 1);          // this thread's window of the item
    const int c0 = t / FG_WIN, c1 = c0 + FG_CAND / 2;
    for (long long item = blockIdx.x; item < total; item += gridDim.x) {
        const int grp = (int)(item % groups), chunk = (int)(item / groups);
        __syncthreads();
        if (t == 0) {
            s_any = 0;
            s_lo = INT_MAX;
            s_hi = -1;
        }
        __syncthreads();
        if (t < FG_CAND) {
            const int li = grp * FG_CAND + t;
            const int pos = li < C ? list[li] : -1;
            cp[t] = pos;
            cw[t] = pos >= 0 ? cand[pos] : 0;
            live[t] = pos >= 0 && !__ldcg(pruned + pos);
            if (live[t]) atomicOr(&s_any, 1);
        }
        if (t < FG_WIN) {
            const int fi = chunk * FG_WIN + t;
            const int f = fi < F ? frag[fi] : -1;
            fw[t] = (f >= col_lo && f < col_hi) ? f : -1;
            if (fw[t] >= 0) {
                atomicMin(&s_lo, f);
                atomicMax(&s_hi, f);
            }
        }
        __syncthreads();
        if (!s_any || s_hi < 0) continue;
        const int lo = s_lo, span = s_hi - s_lo + m;
        const bool staged = span <= FG_SPAN;
        for (int e = t; e < FG_CAND * m; e += FG_THREADS) {
            const int c = e / m, k = e - c * m;
            fg_a[e] = live[c] ? (double)x[cw[c] + k] - mu64[cw[c]] : 0.0;
        }
        if (staged)
            for (int p = t; p < span; p += FG_THREADS) xs[p] = x[lo + p];
        __syncthreads();
        double b0 = -INFINITY, b1 = -INFINITY;
        const int f = fw[wi];
        if (f >= 0 && (live[c0] || live[c1])) {
            const double mf = mu64[f];
            const double *a0 = fg_a + c0 * m, *a1 = fg_a + c1 * m;
            double acc0 = 0.0, acc1 = 0.0;
            if (staged) {
                const float *y = xs + (f - lo);
#pragma unroll 4
                for (int k = 0; k < m; ++k) {
                    const double v = (double)y[k] - mf;
                    acc0 = fma(a0[k], v, acc0);
                    acc1 = fma(a1[k], v, acc1);
                }
            } else {
                const float *y = x + f;
#pragma unroll 8
                for (int k = 0; k < m; ++k) {
                    const double v = (double)__ldg(y + k) - mf;
                    acc0 = fma(a0[k], v, acc0);
                    acc1 = fma(a1[k], v, acc1);
                }
            }
            const double ivf = inv64[f];
            const int d0 = cw[c0] > f ? cw[c0] - f : f - cw[c0];
            const int d1 = cw[c1] > f ? cw[c1] - f : f - cw[c1];
            if (live[c0] && d0 >= m - 1) b0 = acc0 * inv64[cw[c0]] * ivf;
            if (live[c1] && d1 >= m - 1) b1 = acc1 * inv64[cw[c1]] * ivf;
        }
        // maxima over the item's 64 windows: two warps per candidate pair
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            b0 = fmax(b0, __shfl_xor_sync(0xffffffffu, b0, o));
            b1 = fmax(b1, __shfl_xor_sync(0xffffffffu, b1, o));
        }
        if (lane == 0) {
            best_s[c0][warp & 1] = b0;
            best_s[c1][warp & 1] = b1;
        }
        __syncthreads();
        if (t < FG_CAND && live[t]) {
            const double v = fmax(best_s[t][0], best_s[t][1]);
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
    const size_t smem = sizeof(double) * (size_t)FG_CAND * m;
    cudaError_t e = paddi_raise_smem_limit((const void *)k_fragile, smem);
    if (e != cudaSuccess) return e;
    k_fragile<<<num_sms * 4, FG_THREADS, smem, st>>>(x, mu64, inv64, cand, list, list_count,
                                                    pruned, rho_max, frag, frag_count, m, thr,
                                                    col_lo, col_hi);
    return cudaGetLastError();
}
