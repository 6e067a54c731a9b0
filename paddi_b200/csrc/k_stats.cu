// k_stats.cu -- per-length window statistics from FP64 prefix sums.
//
// Replaces the reference's gpu_compute_statistics / gpu_update_statistics
// (src/preprocessing.cuh:12-65: FP32, one-pass E[x^2]-mu^2, chained updates
// from length m-1 to m).  Here every length is computed afresh:
//   * each CTA stages a tile of the series, shifts it by the tile's first
//     value c, and builds inclusive FP64 prefix sums of (x-c) and (x-c)^2 in
//     shared memory (warp-shuffle scans);
//   * window sums are differences of two prefix entries, so the variance
//     never subtracts two numbers of the size of the raw values;
//   * flatness (all m values equal) is an exact integer test on a prefix
//     count of equal neighbours.
// HBM traffic per length: 4 B read + 37 B written per window.
#include <float.h>
#include <limits.h>

#include "paddi_internal.cuh"

namespace {

constexpr int ST_THREADS = 256;
constexpr int ST_TILE = 2048; // windows per CTA (the staged halo of m values is amortised over them)
constexpr int ST_MAXM = 1024; // longest supported window

// dynamic shared memory of one CTA for length m: P1, P2 (FP64 prefixes), E
// (int prefix of equal neighbours) and the staged values, ST_TILE + m + 2 each
__host__ __device__ inline size_t st_smem(int m)
{
    const size_t L = (size_t)ST_TILE + (size_t)m + 2;
    return L * (2 * sizeof(double) + sizeof(int) + sizeof(float));
}

// Exclusive-to-inclusive block scan over `cnt` per-thread partials.
template <typename T>
__device__ T block_exclusive_scan(T v, T *warp_tot)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_tot[w] = inc;
    __syncthreads();
    if (w == 0) {
        T t = lane < (ST_THREADS / 32) ? warp_tot[lane] : T(0);
        T ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += u;
        }
        if (lane < (ST_THREADS / 32)) warp_tot[lane] = ti - t; // exclusive
    }
    __syncthreads();
    T r = warp_tot[w] + inc - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(ST_THREADS)
k_window_stats(const float *__restrict__ x, int64_t n, int32_t m, int32_t N, float4 *wst,
               float *mu, double *mu64, double *inv64, uint8_t *flat, int32_t *flat_count,
               int32_t *flat_span)
{
    // staged values: x[t0 .. t0 + ST_TILE + m] (one extra window for mu_{i+1})
    extern __shared__ __align__(16) unsigned char st_mem[];
    const int LS = ST_TILE + m + 2;
    double *P1 = reinterpret_cast<double *>(st_mem);
    double *P2 = P1 + LS;
    int *E = reinterpret_cast<int *>(P2 + LS);
    float *xs = reinterpret_cast<float *>(E + LS);
    __shared__ double wtot_d[ST_THREADS / 32];
    __shared__ int wtot_i[ST_THREADS / 32];

    const int64_t t0 = (int64_t)blockIdx.x * ST_TILE;
    const int len = ST_TILE + m + 1; // values staged
    const float c = x[t0 < n ? t0 : n - 1];
    for (int k = threadIdx.x; k < len; k += ST_THREADS) {
        const int64_t g = t0 + k;
        xs[k] = g < n ? x[g] : c;
    }
    __syncthreads();
    // per-thread serial chunk, then block scan of chunk totals
    const int per = (len + ST_THREADS - 1) / ST_THREADS;
    const int k0 = threadIdx.x * per;
    double s1 = 0.0, s2 = 0.0;
    int se = 0;
    for (int k = k0; k < k0 + per && k < len; ++k) {
        const double d = (double)xs[k] - (double)c;
        s1 += d;
        s2 += d * d;
        se += (k + 1 < len) ? (xs[k] == xs[k + 1]) : 0;
    }
    double b1 = block_exclusive_scan<double>(s1, wtot_d);
    double b2 = block_exclusive_scan<double>(s2, wtot_d);
    int be = block_exclusive_scan<int>(se, wtot_i);
    // exclusive prefixes: P[k] = sum over staged values < k
    for (int k = k0; k < k0 + per && k < len; ++k) {
        P1[k] = b1;
        P2[k] = b2;
        E[k] = be;
        const double d = (double)xs[k] - (double)c;
        b1 += d;
        b2 += d * d;
        be += (k + 1 < len) ? (xs[k] == xs[k + 1]) : 0;
    }
    if (threadIdx.x == ST_THREADS - 1 || (k0 < len && k0 + per >= len)) {
        P1[len] = b1;
        P2[len] = b2;
        E[len] = be;
    }
    __syncthreads();

    const double invm = 1.0 / (double)m;
    int nflat = 0;
    for (int l = threadIdx.x; l < ST_TILE; l += ST_THREADS) {
        const int64_t i = t0 + l;
        if (i >= (int64_t)N + PADDI_PAD_WIN) break;
        if (i >= N) { // zeroed tail so tiles can over-read
            wst[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            mu[i] = 0.f;
            mu64[i] = 0.0;
            inv64[i] = 0.0;
            flat[i] = 0;
            continue;
        }
        // window i and window i+1
        const double a1 = P1[l + m] - P1[l], a2 = P2[l + m] - P2[l];
        const int fe = (E[l + m - 1] - E[l]) == (m - 1);
        const double um = a1 * invm;
        const double q = a2 - a1 * um;
        const double nrm = fe ? 0.0 : sqrt(q > 0.0 ? q : 0.0);
        const int fl = fe || nrm == 0.0; // flat: zero norm
        const double iv = fl ? 0.0 : 1.0 / nrm;
        const double mu_i = fe ? (double)xs[l] : (double)c + um;
        float df = 0.f, dg = 0.f;
        if (i + 1 < N) {
            const double c1 = P1[l + 1 + m] - P1[l + 1];
            const int fl1 = (E[l + m] - E[l + 1]) == (m - 1);
            const double mu_n = fl1 ? (double)xs[l + 1] : (double)c + c1 * invm;
            const double xe = (double)xs[l + m], xb = (double)xs[l];
            df = (float)((xe - xb) * 0.5);
            dg = (float)((xe - mu_n) + (xb - mu_i));
        }
        wst[i] = make_float4(df, dg, (float)iv, fl ? 0.f : (float)nrm);
        mu[i] = (float)mu_i;
        mu64[i] = mu_i;
        inv64[i] = iv;
        flat[i] = (uint8_t)fl;
        nflat += fl;
        // lowest and highest flat window, both kept as maxima over a zeroed
        // pair: {INT_MAX - lowest, highest + 1} (flat windows are rare)
        if (fl && flat_span) {
            atomicMax(flat_span, INT_MAX - (int)i);
            atomicMax(flat_span + 1, (int)i + 1);
        }
    }
    if (nflat) atomicAdd(flat_count, nflat);
}

// mean / population std in the reference's FP32 layout (src/preprocessing.cuh:31-34)
__global__ void k_export_stats(const double *__restrict__ mu64, const double *__restrict__ inv64,
                               int32_t N, int32_t m, float *mean, float *sd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    mean[i] = (float)mu64[i];
    const double iv = inv64[i];
    sd[i] = iv > 0.0 ? (float)(1.0 / (iv * sqrt((double)m))) : 0.f;
}

} // namespace

cudaError_t paddi_launch_export_stats(const double *mu64, const double *inv64, int32_t N,
                                      int32_t m, float *mean, float *sd, cudaStream_t st)
{
    k_export_stats<<<(N + 255) / 256, 256, 0, st>>>(mu64, inv64, N, m, mean, sd);
    return cudaGetLastError();
}

cudaError_t paddi_launch_stats(const float *x, int64_t n, int32_t m, float4 *wst, float *mu,
                               double *mu64, double *inv64, uint8_t *flat,
                               int32_t *flat_count, cudaStream_t st, int32_t *flat_span)
{
    if (m < 2 || m > ST_MAXM || n < 2 * (int64_t)m) return cudaErrorInvalidValue;
    const int32_t N = (int32_t)(n - m + 1);
    const int64_t total = (int64_t)N + PADDI_PAD_WIN;
    const unsigned grid = (unsigned)((total + ST_TILE - 1) / ST_TILE);
    const size_t smem = st_smem(m);
    cudaError_t e = paddi_raise_smem_limit((const void *)k_window_stats, smem);
    if (e != cudaSuccess) return e;
    k_window_stats<<<grid, ST_THREADS, smem, st>>>(x, n, m, N, wst, mu, mu64, inv64, flat,
                                                   flat_count, flat_span);
    return cudaGetLastError();
}
