// k_refine_fp32.cu -- dense candidate refine on CUDA cores (the plain FP32 form).
//
// Reference: gpu_global_discords_refine (src/PD3_kernels.cuh:582-662): a
// 32x32-tiled SGEMM of the candidate matrix C (m x Cc, gathered on the host)
// with the Hankel windows of the series, the distance formula in the
// epilogue, and a CAS-loop float atomicMin per candidate.
//
// Here:
//   * candidates are an index list produced on the device; each work item
//     is (32 candidates) x (a slice of all windows), pulled from a counter by
//     a persistent grid;
//   * the candidate operand is the z-normalised window z_c = (x_c - mu_c) inv_c,
//     staged once per item; the window operand is the raw series shifted by a
//     per-chunk constant (the shift cancels because sum_k z_c[k] = 0, and the
//     rounding residue is removed with the candidate's FP32 sum of z_c);
//   * every thread holds 4 candidates x 8 windows of accumulators; the 8
//     window operands rotate through a register ring (one shared load per k);
//   * the epilogue forms rho = <z_c, x_j - mu_j> inv_j, applies the
//     trivial-match exclusion |c - j| >= m-1, keeps the running maximum
//     (maximum rho == minimum distance) and flags a candidate as pruned as
//     soon as its correlation with some window exceeds thr (early abandoning:
//     an item stops when all 32 of its candidates are pruned, and later items
//     of a fully pruned tile are skipped);
//   * one atomicMax per candidate per item on an order-preserving integer
//     image of rho (no CAS loop).
// Rounding: the dot products are summed in two levels (blocks of 64 terms),
// so a correlation with window j is within g_j = window_bound(E, A_j) of the
// exact one, A_j the amplification |x_j - sh| / |x_j - mu_j| of the chunk's
// shift.  Windows with g_j above gcap are fragile: their correlations are
// lowered by their own g_j (a safe lower bound to prune on) and they are
// evaluated in FP64 by the fragile pass.  The chunk's largest other g_j, G,
// is subtracted from the other correlations for the prune test, and added
// back to the kept maxima, so those are the middle of an interval of
// half-width at most gcap (a fragile window's lowered value never exceeds its
// true one).  Chunks start
// at multiples of 256 windows, so the fragile set depends only on the length.
#include <float.h>

#include <cmath>

#include "paddi_internal.cuh"

using paddi::f2ord;

namespace {

constexpr int RF_THREADS = 256; // 8 warps x 4 candidates
constexpr int RF_TC = 32;       // candidates per item
constexpr int RF_TW = 256;      // windows per chunk (32 lanes x 8)
static_assert(RF_TW == RF_THREADS, "one window of the chunk per thread at staging");
constexpr int RF_MAXM = 1024;

__device__ __forceinline__ int xpad(int p) { return p + (p >> 5); }

struct RfSmem {
    float *zT;    // [mpad][RF_TC]
    float *xs;    // xpad(RF_TW + mpad + 8)
    float *cinv;  // [RF_TW]
    float *cmu;   // [RF_TW]
    float *cflt;  // [RF_TW]
    float *cgm;   // [RF_TW]: the bound subtracted from each window's correlations
};

constexpr int RF_SUMBLK = 64; // two-level sums: terms per partial sum

__global__ void __launch_bounds__(RF_THREADS)
k_refine_fp32(const float *__restrict__ x, const float4 *__restrict__ wst,
              const float *__restrict__ mu, const int32_t *__restrict__ cand,
              const int32_t *__restrict__ list, const int32_t *__restrict__ list_count,
              PaddiAttemptDev *att, int32_t *work, uint32_t *rho_max, uint8_t *pruned, int32_t N,
              int32_t m, int32_t jb, int32_t je, float thr, int32_t grid_ctas, float E,
              float gcap)
{
    extern __shared__ __align__(16) unsigned char rf_smem[];
    const int mpad = (m + 7) & ~7;
    RfSmem S;
    S.zT = reinterpret_cast<float *>(rf_smem);
    S.xs = S.zT + (size_t)mpad * RF_TC;
    S.cinv = S.xs + xpad(RF_TW + mpad + 8) + 4;
    S.cmu = S.cinv + RF_TW;
    S.cflt = S.cmu + RF_TW;
    S.cgm = S.cflt + RF_TW;
    __shared__ int s_item, s_alive;
    __shared__ float s_gred[RF_THREADS / 32];
    __shared__ int cw[RF_TC], cp[RF_TC];
    __shared__ float cf[RF_TC], zsum[RF_TC];
    __shared__ uint8_t dead[RF_TC];

    const int C = *list_count;
    if (C <= 0 || je <= jb) return;
    const int range = je - jb;
    const int tiles = (C + RF_TC - 1) / RF_TC;
    int splits = (2 * grid_ctas + tiles - 1) / tiles;
    const int max_splits = max(1, range / (4 * RF_TW));
    splits = max(1, min(splits, max_splits));
    const int span = (((range + splits - 1) / splits) + RF_TW - 1) / RF_TW * RF_TW;
    const int total = tiles * splits;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(work, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;
        const int tile = item % tiles, split = item / tiles;
        // ---- candidates of this item
        if (threadIdx.x < RF_TC) {
            const int li = tile * RF_TC + threadIdx.x;
            const bool v = li < C;
            const int pos = v ? list[li] : 0;
            const int w = v ? cand[pos] : 0;
            cw[threadIdx.x] = w;
            cp[threadIdx.x] = pos;
            dead[threadIdx.x] = !v || __ldcg(pruned + pos);
            cf[threadIdx.x] = (v && wst[w].z == 0.f) ? 1.f : 0.f; // flat candidate
        }
        __syncthreads();
        int alive = 0;
        if (threadIdx.x < RF_TC) alive = !dead[threadIdx.x];
        if (!__syncthreads_or(alive)) continue;
        // ---- z-normalised candidate windows, k-major
        for (int e = threadIdx.x; e < mpad * RF_TC; e += RF_THREADS) {
            const int c = e & (RF_TC - 1), k = e >> 5;
            float z = 0.f;
            if (k < m && !dead[c]) {
                const int w = cw[c];
                z = (x[w + k] - mu[w]) * wst[w].z;
            }
            S.zT[e] = z;
        }
        __syncthreads();
        if (threadIdx.x < RF_TC) { // two-level sum of the candidate's z
            float s = 0.f;
            for (int k0 = 0; k0 < m; k0 += RF_SUMBLK) {
                float p = 0.f;
                for (int k = k0; k < min(m, k0 + RF_SUMBLK); ++k) p += S.zT[k * RF_TC + threadIdx.x];
                s += p;
            }
            zsum[threadIdx.x] = s;
        }
        const int j_lo = jb + split * span, j_hi = min(je, j_lo + span);
        float rmax[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (int j0 = j_lo; j0 < j_hi; j0 += RF_TW) {
            __syncthreads();
            const float sh = x[j0];
            for (int p = threadIdx.x; p < RF_TW + mpad + 8; p += RF_THREADS) {
                const int g = j0 + p;
                S.xs[xpad(p)] = (g < N + m - 1 ? x[g] : sh) - sh;
            }
            // one window per thread (RF_TW == RF_THREADS): its bound, fragile or not
            const int qt = threadIdx.x;
            const float4 wsq = wst[j0 + qt]; // zero beyond N
            const float mq = mu[j0 + qt];
            const float gt = paddi::window_bound(wsq.z, mq, sh, (float)m, E, 0.f);
            const bool fragt = j0 + qt < N && gt > gcap;
            S.cinv[qt] = wsq.z;
            S.cflt[qt] = wsq.z == 0.f ? 1.f : 0.f; // flat window (or the padded tail)
            S.cmu[qt] = mq;
            float gq = fragt ? 0.f : gt; // the chunk's largest bound over its non-fragile windows
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) gq = fmaxf(gq, __shfl_xor_sync(0xffffffffu, gq, o));
            if (lane == 0) s_gred[warp] = gq;
            __syncthreads();
            float G = 0.f;
#pragma unroll
            for (int w2 = 0; w2 < RF_THREADS / 32; ++w2) G = fmaxf(G, s_gred[w2]);
            S.cgm[qt] = fragt ? gt : G;
            __syncthreads();
            float acc[4][8], tot[4][8];
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) acc[c][jj] = tot[c][jj] = 0.f;
            float ring[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) ring[jj] = S.xs[xpad(8 * lane + jj)];
            const float4 *z4 = reinterpret_cast<const float4 *>(S.zT) + warp;
            for (int k0 = 0; k0 < mpad; k0 += 8) {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const float4 z = z4[(k0 + u) * (RF_TC / 4)];
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) {
                        const float xv = ring[(u + jj) & 7];
                        acc[0][jj] = fmaf(z.x, xv, acc[0][jj]);
                        acc[1][jj] = fmaf(z.y, xv, acc[1][jj]);
                        acc[2][jj] = fmaf(z.z, xv, acc[2][jj]);
                        acc[3][jj] = fmaf(z.w, xv, acc[3][jj]);
                    }
                    ring[u] = S.xs[xpad(8 * lane + k0 + u + 8)];
                }
                if (((k0 + 8) & (RF_SUMBLK - 1)) == 0 || k0 + 8 >= mpad) {
#pragma unroll
                    for (int c = 0; c < 4; ++c)
#pragma unroll
                        for (int jj = 0; jj < 8; ++jj) {
                            tot[c][jj] += acc[c][jj];
                            acc[c][jj] = 0.f;
                        }
                }
            }
            // ---- epilogue
            bool hit[4] = {false, false, false, false};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int ci = 4 * warp + c;
                const int w = cw[ci];
                const float zs = zsum[ci], fc = cf[ci];
                float cmax = -INFINITY;
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    const int q = 8 * lane + jj;
                    const int j = j0 + q;
                    const int dd = w > j ? w - j : j - w;
                    const bool ok = (j < j_hi) && (dd >= m - 1);
                    // lower bound of the correlation (NaN for a fragile window)
                    const float rho = fmaf(fmaf(-zs, S.cmu[q] - sh, tot[c][jj]), S.cinv[q],
                                           fmaf(fc, S.cflt[q], -S.cgm[q]));
                    if (ok) {
                        cmax = fmaxf(cmax, rho);
                        hit[c] |= rho > thr;
                    }
                }
                rmax[c] = fmaxf(rmax[c], cmax + G); // the interval's middle
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int ci = 4 * warp + c;
                if (__any_sync(0xffffffffu, hit[c]) && lane == 0 && !dead[ci]) {
                    dead[ci] = 1;
                    pruned[cp[ci]] = 1;
                }
            }
            __syncthreads();
            // early abandon: stop once every candidate of the item is pruned
            if (threadIdx.x == 0) s_alive = 0;
            __syncthreads();
            if (threadIdx.x < RF_TC) {
                if (!dead[threadIdx.x] && __ldcg(pruned + cp[threadIdx.x])) dead[threadIdx.x] = 1;
                if (!dead[threadIdx.x]) s_alive = 1;
            }
            if (threadIdx.x == 0) atomicAdd(&att->n_pairs, (unsigned long long)(RF_TC * RF_TW));
            __syncthreads();
            if (!s_alive) break;
        }
        // ---- fold the item's maxima into the global ones
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float v = rmax[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            const int ci = 4 * warp + c;
            if (lane == 0 && tile * RF_TC + ci < C && v > -INFINITY)
                atomicMax(rho_max + cp[ci], f2ord(v));
        }
        __syncthreads();
    }
}

} // namespace

cudaError_t paddi_launch_refine_fp32(const float *x, const float4 *wst, const float *mu,
                                     const int32_t *cand, const int32_t *list,
                                     const int32_t *list_count, PaddiAttemptDev *att,
                                     int32_t *work, uint32_t *rho_max, uint8_t *pruned,
                                     int32_t N, int32_t m, int32_t jb, int32_t je, float thr,
                                     float gcap, int32_t num_sms, cudaStream_t st)
{
    if (m > RF_MAXM) return cudaErrorInvalidValue;
    if ((jb % RF_TW) != 0) return cudaErrorInvalidValue; // chunks on the 256-window grid
    const int mpad = (m + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)mpad * RF_TC + (RF_TW + mpad + 8) +
                                         ((RF_TW + mpad + 8) >> 5) + 4 + 4 * RF_TW) + 16;
    cudaError_t e = paddi_raise_smem_limit((const void *)k_refine_fp32, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_refine_fp32, RF_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = num_sms * per_sm;
    k_refine_fp32<<<grid, RF_THREADS, smem, st>>>(x, wst, mu, cand, list, list_count, att, work,
                                                  rho_max, pruned, N, m, jb, je, thr, grid,
                                                  paddi_bound_fp32(m).E, gcap);
    return cudaGetLastError();
}

PaddiBound paddi_bound_fp32(int m)
{
    const double u = std::ldexp(1.0, -24);
    const int mpad = (m + 7) & ~7;
    // the dot product in two levels (64 terms, then mpad/64 partials), the z
    // sum likewise, z's own rounding (x - mu, times inv: 3u), the shifted slice
    // (u), the epilogue (4u), the FP32 rounding of thr (2u)
    const double dot = (double)RF_SUMBLK + std::ceil(mpad / (double)RF_SUMBLK) + 1.0;
    PaddiBound B;
    B.E = (float)((2.0 * dot + 10.0) * u * 1.01);
    B.F = 0.f;
    return B;
}

// Fragile windows of length m for the FP32 refine's geometry (chunks of 256
// windows shifted by their first value): the same test as the refine applies.
__global__ void k_fragile_scan_fp32(const float *__restrict__ x, const float4 *__restrict__ wst,
                                    const float *__restrict__ mu, int32_t N, int32_t m, float E,
                                    float gcap, int32_t *frag_list, int32_t *frag_count)
{
    const int lane = threadIdx.x & 31;
    for (int j0 = blockIdx.x * blockDim.x; j0 < N; j0 += gridDim.x * blockDim.x) {
        const int j = j0 + threadIdx.x;
        bool frag = false;
        if (j < N) {
            const float sh = x[j & ~(RF_TW - 1)];
            frag = paddi::window_bound(wst[j].z, mu[j], sh, (float)m, E, 0.f) > gcap;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, frag);
        if (bal) {
            int base = 0;
            if (lane == 0) base = atomicAdd(frag_count, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (frag) frag_list[base + __popc(bal & ((1u << lane) - 1u))] = j;
        }
    }
}

cudaError_t paddi_launch_fragile_scan_fp32(const float *x, const float4 *wst, const float *mu,
                                           int32_t N, int32_t m, float gcap, int32_t *frag_list,
                                           int32_t *frag_count, int32_t num_sms, cudaStream_t st)
{
    k_fragile_scan_fp32<<<num_sms * 4, 256, 0, st>>>(x, wst, mu, N, m, paddi_bound_fp32(m).E, gcap,
                                                    frag_list, frag_count);
    return cudaGetLastError();
}
