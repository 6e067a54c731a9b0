// k_guide.cu -- exact FP64 nearest-neighbour distance of the r policy's bound
// window, kept incrementally across lengths.
//
// (No counterpart in the reference: its r schedule, src/main.cu:136-233,
// uses no bound.)  The BOUND and LEARNED policies start length m from the
// exact nn, at length m, of the previous length's top-1 window w: the top-1
// distance is the largest nn, so it is a lower bound.  The nn is a minimum
// over the admissible windows j of 2m (1 - rho(w, j)), and rho needs the
// centred dot product of w with every j.  The shifted dot products
//     G[j] = sum_{k<m} (x[w+k] - s) (x[j+k] - s)
// change by a few terms from one length to the next: the top-1 window of
// the next length is mostly w again, or a window a few places away (a
// discord centred on an anomaly starts one place earlier when the length
// grows by one).  For w' = w + delta at length m + 1, pairing the same
// partner offset j - w,
//     G'[j] = G[j - delta] + (terms of [w', w'+m+1) not in [w, w+m))
//                          - (terms of [w, w+m) not in [w', w'+m+1)),
// |delta| + |delta + 1| FMA per window instead of m; a slide is taken while
// that is at most m/4 (and |delta| <= 32).  The centred product is
//     cov(w, j) = G[j] - A (mu_j - s),   A = sum_{k<m} (x[w+k] - s),
// with A summed from the series in FP64 at every launch: writing it as
// m (mu_w - s) would carry the rounding of the FP64 mean, times |mu_j - s|
// (series levels far apart), into every correlation -- about 1e-10 relative
// on a random walk, enough to round a reported distance to the neighbouring
// float.
// The shift s is w's mean at the length G was built for, so the shifted
// values stay of the order of the local range of the series; G is rebuilt
// with direct dot products after 64 slides, when the window moves further,
// and when the state belongs to another length.
//
// Two kernels are queued per length.  Both read the window (from the host,
// or from the previous attempt's result on the device, so they can be queued
// before the host has seen that result) and compare it with the state of G.
// k_guide_stream reuses G (same window and length) or slides it into the
// other buffer: a streaming pass with no large shared memory, four windows
// per thread and step so their loads are in flight together.  k_guide_build
// then rebuilds G with direct dot products staged in shared memory, but only
// if the state was left untouched, i.e. when the first kernel found a
// rebuild due.  Windows whose old partner entry does not exist (|delta| at
// most, at the ends of the series) are summed directly, one per CTA.  In
// each kernel the last CTA to finish publishes the new state, after every
// CTA has read the old one.
#include <float.h>

#include <algorithm>

#include "paddi_internal.cuh"

using paddi::d2ord;

namespace {

constexpr int GD_THREADS = 256;
constexpr int GD_JPT = 8;                          // windows per thread (build)
constexpr int GD_SPAN = GD_THREADS * GD_JPT;       // windows per build item
constexpr int GD_MAXM = 1024;
constexpr int GD_MAX_AGE = 64;                     // slides before a rebuild
constexpr int GD_MAX_SLIDE = 32;                   // largest |delta| of a slide
constexpr int GD_STREAM_CTAS_PER_SM = 4;          // one wave at <= 64 registers
constexpr int GD_UNROLL = 4;                       // windows per thread and step (stream)

__device__ __forceinline__ int gpad(int d) { return d + (d >> 4); } // conflict-free at stride 8

__device__ __forceinline__ bool admissible(int w, int j, int m)
{
    const int d = w > j ? w - j : j - w;
    return d >= m - 1;
}

// 2m (1 - rho) of (w, j) from the centred dot product, with the flat-window
// policy of the selection (one flat window: rho 0; two: rho 1).
__device__ __forceinline__ double pair_dist(double cov, double iw, double ij, int fw, int fj, int m)
{
    double rho;
    if (fw | fj) rho = (fw & fj) ? 1.0 : 0.0;
    else rho = cov * iw * ij;
    const double d = 2.0 * m * (1.0 - rho);
    return d < 0.0 ? 0.0 : d;
}

// Block-wide sum (all threads get it); red holds one double per warp.
__device__ __forceinline__ double block_sum(double v, double *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int q = 0; q < GD_THREADS / 32; ++q) t += red[q];
    return t;
}

// The window of this length: w_host, or the top-1 window of the previous
// attempt's result (-1: none), clamped to the last window.
__device__ __forceinline__ int guide_window(const PaddiAttemptResult *prev, int w_host, int N)
{
    int w = w_host;
    if (w < 0) w = (prev->status == 0 && prev->n_sel > 0) ? prev->sel_ind[0] : -1;
    if (w >= N) w = N - 1;
    return w;
}

__device__ __forceinline__ int guide_mode(const PaddiGuide *g, int w, int m)
{
    const int gm = g->m, delta = w - g->w;
    if (gm > 0 && delta == 0 && gm == m) return PADDI_GUIDE_REUSED;
    if (gm > 0 && gm == m - 1 && delta >= -GD_MAX_SLIDE && delta <= GD_MAX_SLIDE &&
        4 * (abs(delta) + abs(delta + 1)) <= m && g->age < GD_MAX_AGE)
        return PADDI_GUIDE_SLID;
    return PADDI_GUIDE_BUILT;
}

// Grid minimum into g->nn_ord; the last CTA to arrive publishes the state.
__device__ __forceinline__ void guide_finish(double best, double *red, PaddiGuide *g, int w, int m,
                                             double s, int cur, int age, int mode)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = INFINITY;
        for (int q = 0; q < GD_THREADS / 32; ++q) b = fmin(b, red[q]);
        if (b < INFINITY) atomicMin(&g->nn_ord, d2ord(b));
        __threadfence();
        if (atomicAdd(&g->done, 1) == (int)gridDim.x - 1) {
            g->w = w;
            g->m = m;
            g->s = s;
            g->cur = cur;
            g->age = age;
            g->w_used = w;
            g->mode = mode;
            g->done = 0;
            g->item = 0;
        }
    }
}

// Reuse and slide.  Leaves without a trace when a rebuild is due.
__global__ void __launch_bounds__(GD_THREADS, GD_STREAM_CTAS_PER_SM)
k_guide_stream(const float *__restrict__ x, const double *__restrict__ mu64,
               const double *__restrict__ inv64, const uint8_t *__restrict__ flat, int32_t N,
               int32_t m, const PaddiAttemptResult *__restrict__ prev, int32_t w_host,
               PaddiGuide *g, double *__restrict__ G0, double *__restrict__ G1)
{
    __shared__ double redm[GD_THREADS / 32];
    __shared__ double cf[2 * GD_MAX_SLIDE + 2]; // slide coefficients, signed
    __shared__ int coff[2 * GD_MAX_SLIDE + 2];  // their partner offsets (from j)
    const int t = threadIdx.x;
    const int w = guide_window(prev, w_host, N);
    if (w < 0) { // no top-1 window: nothing to bound with, the state stays
        if (blockIdx.x == 0 && t == 0) {
            g->w_used = -1;
            g->mode = PADDI_GUIDE_SKIPPED;
        }
        return;
    }
    const int mode = guide_mode(g, w, m);
    if (mode == PADDI_GUIDE_BUILT) return; // k_guide_build's turn
    const int gw = g->w, gm = g->m, gcur = g->cur, gage = g->age;
    const int delta = w - gw;
    const double s = g->s;
    const double *Gin = gcur ? G1 : G0;
    double *Gout = gcur ? G0 : G1; // slide only
    const double iw = inv64[w];
    const int fw = flat[w];
    double cw = 0.0; // A: cov = G[j] - A (mu_j - s)
    for (int k = t; k < m; k += GD_THREADS) cw += (double)x[w + k] - s;
    cw = block_sum(cw, redm);
    double best = INFINITY;

    // ---- the slide's terms: [w, w+m) against the old [gw, gw+gm).  The two
    //      ranges overlap (|delta| < m), so the terms are the values between
    //      the two starts, [f0, f0+nf) (added when w < gw, else removed), and
    //      between the two ends, [e0, e0+ne) (added when the new end is
    //      later); their signed, shifted values go to cf, their offsets
    //      from the partner window's start to coff
    int nf = 0, ne = 0, f0 = 0, e0 = 0;
    int blo = 0, bhi = N; // windows without an old partner entry: [0, blo) and [bhi, N)
    if (mode == PADDI_GUIDE_SLID) {
        f0 = min(w, gw);
        nf = max(w, gw) - f0;
        const double fs = w < gw ? 1.0 : -1.0;
        const int a1 = w + m, b1 = gw + gm;
        e0 = min(a1, b1);
        ne = max(a1, b1) - e0;
        const double es = a1 > b1 ? 1.0 : -1.0;
        for (int k = t; k < nf + ne; k += GD_THREADS) {
            const int q = k < nf ? f0 + k : e0 + k - nf;
            cf[k] = (k < nf ? fs : es) * ((double)x[q] - s);
            coff[k] = q - w;
        }
        blo = delta > 0 ? delta : 0;
        bhi = min(N, N + 1 + delta); // old entries exist for j - delta < N + 1
        // windows without an old entry: direct sums, one per CTA
        const int nb = blo + (N - bhi);
        if ((int)blockIdx.x < nb) {
            const int jj = (int)blockIdx.x < blo ? (int)blockIdx.x : bhi + (int)blockIdx.x - blo;
            double v = 0.0;
            for (int k = t; k < m; k += GD_THREADS)
                v = fma((double)x[w + k] - s, (double)x[jj + k] - s, v);
            v = block_sum(v, redm);
            if (t == 0) Gout[jj] = v;
            if (admissible(w, jj, m)) {
                const double cov = v - cw * (mu64[jj] - s);
                best = fmin(best, pair_dist(cov, iw, inv64[jj], fw, flat[jj], m));
            }
        }
    }
    __syncthreads(); // cf, coff staged
    // ---- streaming pass over the windows with an old entry: GD_UNROLL
    //      windows a stride apart per thread and step, their loads issued
    //      together (the pass is bound by load latency, not bandwidth)
    const int stride = gridDim.x * GD_THREADS;
    const int nt = nf + ne;
    const int shift = mode == PADDI_GUIDE_SLID ? delta : 0;
    for (int j0 = blo + blockIdx.x * GD_THREADS + t; j0 < bhi; j0 += GD_UNROLL * stride) {
        double gv[GD_UNROLL], mv[GD_UNROLL], iv[GD_UNROLL];
        int fv[GD_UNROLL];
#pragma unroll
        for (int u = 0; u < GD_UNROLL; ++u) {
            const int j = j0 + u * stride;
            const bool ok = j < bhi;
            gv[u] = ok ? Gin[j - shift] : 0.0;
            mv[u] = ok ? mu64[j] : 0.0;
            iv[u] = ok ? inv64[j] : 0.0;
            fv[u] = ok ? flat[j] : 0;
        }
        for (int k = 0; k < nt; ++k) {
            const double c = cf[k];
            const int o = coff[k];
#pragma unroll
            for (int u = 0; u < GD_UNROLL; ++u) {
                const int j = j0 + u * stride;
                if (j < bhi) gv[u] = fma(c, (double)x[j + o] - s, gv[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < GD_UNROLL; ++u) {
            const int j = j0 + u * stride;
            if (j < bhi) {
                if (mode == PADDI_GUIDE_SLID) Gout[j] = gv[u];
                if (admissible(w, j, m)) {
                    const double cov = gv[u] - cw * (mv[u] - s);
                    best = fmin(best, pair_dist(cov, iw, iv[u], fw, fv[u], m));
                }
            }
        }
    }
    const bool slid = mode == PADDI_GUIDE_SLID;
    guide_finish(best, redm, g, w, m, s, slid ? gcur ^ 1 : gcur, gage + (slid ? 1 : 0), mode);
}

// Rebuild: direct dot products of w with blocks of GD_SPAN windows, handed
// out dynamically; each thread owns GD_JPT consecutive windows and slides a
// register ring over the staged series.  Leaves when the state is current
// (k_guide_stream did this length) or there is no window.
__global__ void __launch_bounds__(GD_THREADS)
k_guide_build(const float *__restrict__ x, const double *__restrict__ mu64,
              const double *__restrict__ inv64, const uint8_t *__restrict__ flat, int32_t N,
              int32_t m, const PaddiAttemptResult *__restrict__ prev, int32_t w_host,
              PaddiGuide *g, double *__restrict__ G0, double *__restrict__ G1)
{
    __shared__ double a[GD_MAXM];
    __shared__ double xs[GD_SPAN + GD_MAXM + (GD_SPAN + GD_MAXM) / 16 + 16];
    __shared__ double redm[GD_THREADS / 32];
    __shared__ int s_item;
    const int t = threadIdx.x;
    const int w = guide_window(prev, w_host, N);
    if (w < 0 || guide_mode(g, w, m) != PADDI_GUIDE_BUILT) return;
    const int ncur = g->cur ^ 1;
    double *Gout = ncur ? G1 : G0;
    const double s = mu64[w];
    const double iw = inv64[w];
    const int fw = flat[w];
    double cw = 0.0; // A: s is w's FP64 mean, so A is only its rounding residue
    for (int k = t; k < m; k += GD_THREADS) {
        a[k] = (double)x[w + k] - s;
        cw += a[k];
    }
    cw = block_sum(cw, redm);
    double best = INFINITY;
    const int nblk = (N + GD_SPAN - 1) / GD_SPAN;
    for (;;) {
        __syncthreads(); // a[] staged; xs free for the next block
        if (t == 0) s_item = atomicAdd(&g->item, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= nblk) break;
        const int j0 = item * GD_SPAN;
        for (int p = t; p < GD_SPAN + m + GD_JPT; p += GD_THREADS) {
            const int q = j0 + p;
            xs[gpad(p)] = (q < N + m - 1 ? (double)x[q] : 0.0) - s;
        }
        __syncthreads();
        const int q0 = GD_JPT * t;
        double acc[GD_JPT], ring[GD_JPT];
#pragma unroll
        for (int c = 0; c < GD_JPT; ++c) {
            acc[c] = 0.0;
            ring[c] = xs[gpad(q0 + c)];
        }
        for (int k0 = 0; k0 < m; k0 += GD_JPT) {
#pragma unroll
            for (int u = 0; u < GD_JPT; ++u) {
                if (k0 + u < m) {
                    const double ak = a[k0 + u];
#pragma unroll
                    for (int c = 0; c < GD_JPT; ++c)
                        acc[c] = fma(ak, ring[(u + c) & (GD_JPT - 1)], acc[c]);
                }
                ring[u] = xs[gpad(q0 + k0 + u + GD_JPT)];
            }
        }
#pragma unroll
        for (int c = 0; c < GD_JPT; ++c) {
            const int j = j0 + q0 + c;
            if (j < N) {
                Gout[j] = acc[c];
                if (admissible(w, j, m)) {
                    const double cov = acc[c] - cw * (mu64[j] - s);
                    best = fmin(best, pair_dist(cov, iw, inv64[j], fw, flat[j], m));
                }
            }
        }
    }
    guide_finish(best, redm, g, w, m, s, ncur, 0, PADDI_GUIDE_BUILT);
}

} // namespace

cudaError_t paddi_launch_guide(const float *x, const double *mu64, const double *inv64,
                               const uint8_t *flat, int32_t N, int32_t m,
                               const PaddiAttemptResult *prev, int32_t w_host, PaddiGuide *g,
                               double *G, size_t g_stride, int32_t num_sms, cudaStream_t st)
{
    if (m < 3 || m > GD_MAXM || N < 1 || g_stride < (size_t)N) return cudaErrorInvalidValue;
    // the result's ordered image starts at +inf (all ones: above every finite
    // image); the rest of the record is written by the kernels
    cudaError_t e = cudaMemsetAsync(&g->nn_ord, 0xff, sizeof(g->nn_ord), st);
    if (e != cudaSuccess) return e;
    // the stream grid also covers the slide's boundary windows (one per CTA)
    const int sgrid = std::max(GD_STREAM_CTAS_PER_SM * num_sms, GD_MAX_SLIDE + 1);
    k_guide_stream<<<sgrid, GD_THREADS, 0, st>>>(x, mu64, inv64, flat, N, m, prev, w_host, g, G,
                                                 G + g_stride);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_guide_build<<<4 * num_sms, GD_THREADS, 0, st>>>(x, mu64, inv64, flat, N, m, prev, w_host,
                                                      g, G, G + g_stride);
    return cudaGetLastError();
}
