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
//     soon as rho > thr_prune (early abandoning: an item stops when all 32 of
//     its candidates are pruned, and later items of a fully pruned tile are
//     skipped);
//   * one atomicMax per candidate per item on an order-preserving integer
//     image of rho (no CAS loop).
#include <float.h>

#include "paddi_internal.cuh"

using paddi::f2ord;

namespace {

constexpr int RF_THREADS = 256; // 8 warps x 4 candidates
constexpr int RF_TC = 32;       // candidates per item
constexpr int RF_TW = 256;      // windows per chunk (32 lanes x 8)
constexpr int RF_MAXM = 1024;

__device__ __forceinline__ int xpad(int p) { return p + (p >> 5); }

struct RfSmem {
    float *zT;    // [mpad][RF_TC]
    float *xs;    // xpad(RF_TW + mpad + 8)
    float *cinv;  // [RF_TW]
    float *cmu;   // [RF_TW]
    float *cflt;  // [RF_TW]
};

__global__ void __launch_bounds__(RF_THREADS)
k_refine_fp32(const float *__restrict__ x, const float4 *__restrict__ wst,
              const float *__restrict__ mu, const int32_t *__restrict__ cand,
              const int32_t *__restrict__ list, const int32_t *__restrict__ list_count,
              PaddiAttemptDev *att, uint32_t *rho_max, uint8_t *pruned, int32_t N, int32_t m,
              int32_t jb, int32_t je, float thr, int32_t grid_ctas)
{
    extern __shared__ __align__(16) unsigned char rf_smem[];
    const int mpad = (m + 7) & ~7;
    RfSmem S;
    S.zT = reinterpret_cast<float *>(rf_smem);
    S.xs = S.zT + (size_t)mpad * RF_TC;
    S.cinv = S.xs + xpad(RF_TW + mpad + 8) + 4;
    S.cmu = S.cinv + RF_TW;
    S.cflt = S.cmu + RF_TW;
    __shared__ int s_item, s_alive;
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
        if (threadIdx.x == 0) s_item = atomicAdd(&att->work_next, 1);
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
        if (threadIdx.x < RF_TC) {
            float s = 0.f;
            for (int k = 0; k < m; ++k) s += S.zT[k * RF_TC + threadIdx.x];
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
            for (int q = threadIdx.x; q < RF_TW; q += RF_THREADS) {
                const float4 ws = wst[j0 + q]; // zero beyond N
                S.cinv[q] = ws.z;
                S.cflt[q] = ws.z == 0.f ? 1.f : 0.f; // flat window (or the padded tail)
                S.cmu[q] = mu[j0 + q];
            }
            __syncthreads();
            float acc[4][8];
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) acc[c][jj] = 0.f;
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
            }
            // ---- epilogue
            bool hit[4] = {false, false, false, false};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int ci = 4 * warp + c;
                const int w = cw[ci];
                const float zs = zsum[ci], fc = cf[ci];
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    const int q = 8 * lane + jj;
                    const int j = j0 + q;
                    const int dd = w > j ? w - j : j - w;
                    const bool ok = (j < j_hi) && (dd >= m - 1);
                    const float rho =
                        fmaf(fmaf(-zs, S.cmu[q] - sh, acc[c][jj]), S.cinv[q], fc * S.cflt[q]);
                    if (ok) {
                        rmax[c] = fmaxf(rmax[c], rho);
                        hit[c] |= rho > thr;
                    }
                }
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
                                     uint32_t *rho_max, uint8_t *pruned, int32_t N, int32_t m,
                                     int32_t jb, int32_t je, float thr_prune, int32_t num_sms,
                                     cudaStream_t st)
{
    if (m > RF_MAXM) return cudaErrorInvalidValue;
    const int mpad = (m + 7) & ~7;
    const size_t smem = sizeof(float) * ((size_t)mpad * RF_TC + (RF_TW + mpad + 8) +
                                         ((RF_TW + mpad + 8) >> 5) + 4 + 3 * RF_TW) + 16;
    cudaError_t e = paddi_raise_smem_limit((const void *)k_refine_fp32, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_refine_fp32, RF_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = num_sms * per_sm;
    k_refine_fp32<<<grid, RF_THREADS, smem, st>>>(x, wst, mu, cand, list, list_count, att, rho_max,
                                                  pruned, N, m, jb, je, thr_prune, grid);
    return cudaGetLastError();
}
