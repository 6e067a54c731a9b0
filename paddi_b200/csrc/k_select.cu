// k_select.cu -- candidate compaction, classification, FP64 recheck and
// top-k selection for one (m, r) attempt.
//
// Reference counterparts:
//   get_node_candidates_num / local_candidates_union (src/sets_processing.hpp:49-113)
//       -> k_compact: warp-scan / block-scan compaction of alive windows
//          into an index list, on the device (no host round trip, no copy of
//          candidate windows: the refine re-reads them from the series);
//   get_node_discords_num / find_top1_discord (src/sets_processing.hpp:11-87)
//       -> k_finalize + k_select: counts of windows with nn >= r^2 and
//          nn > r^2, greedy top-k by nn (first maximum wins);
//   (no counterpart) k_recheck: exact FP64 nearest-neighbour distance of the
//       few windows whose FP32 value lies within the guard band of r^2 or of
//       the top-k cut-off, so the selected set and the reported distances do
//       not depend on FP32 rounding.
#include <float.h>
#include <limits.h>

#include "paddi_internal.cuh"

using paddi::d2ord;
using paddi::f2ord;
using paddi::ord2d;
using paddi::ord2f;

namespace {

constexpr int CP_THREADS = 1024;
constexpr int FZ_THREADS = 1024;
constexpr int RC_THREADS = 256;
constexpr int RC_MAXM = 1024;

// ---------------------------------------------------------------- compact
// Each thread tests 16 consecutive windows (one 16-byte load of alive flags);
// a warp scan and a block scan place them, with one atomicAdd per CTA.
// With prune_flats (r^2 > 0), a flat window that has another flat window at
// least m-1 away is no candidate: their distance is exactly 0 < r^2 under the
// flat-window policy (src/PD3_kernels.cuh:107-108 maps 0/0 to "closer than
// any r").  Phase 1 leaves flat-flat pairs out (rho 0 there), so this is
// where such windows are dropped; the span {INT_MAX - lowest, highest + 1}
// of the flat windows decides it per window.
constexpr int CP_WIN = 16;                 // windows per thread
constexpr int CP_CTHREADS = 256;
__global__ void __launch_bounds__(CP_CTHREADS)
k_compact(const uint8_t *__restrict__ alive, int32_t N, int32_t *cand, uint32_t *rho_max,
          uint8_t *pruned, int32_t *rc_slot, PaddiAttemptDev *att,
          const uint8_t *__restrict__ flat, const int32_t *__restrict__ flat_span, int32_t m,
          int32_t prune_flats)
{
    __shared__ int wcnt[CP_CTHREADS / 32];
    __shared__ int base;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i0 = (blockIdx.x * CP_CTHREADS + threadIdx.x) * CP_WIN;
    uint8_t f[CP_WIN];
    if (i0 + CP_WIN <= N) {
        const uint4 v = *reinterpret_cast<const uint4 *>(alive + i0);
        const uint32_t u[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int b = 0; b < CP_WIN; ++b) f[b] = (u[b >> 2] >> (8 * (b & 3))) & 0xffu;
    } else {
#pragma unroll
        for (int b = 0; b < CP_WIN; ++b) f[b] = i0 + b < N ? alive[i0 + b] : 0;
    }
    uint32_t mask = 0;
    int lo = 0, hi = -1;
    if (prune_flats) {
        lo = INT_MAX - flat_span[0];
        hi = flat_span[1] - 1;
    }
#pragma unroll
    for (int b = 0; b < CP_WIN; ++b) {
        bool a = f[b] != 0;
        const int i = i0 + b;
        if (a && prune_flats && flat[i] && (i - lo >= m - 1 || hi - i >= m - 1)) a = false;
        mask |= (uint32_t)a << b;
    }
    const int cnt = __popc(mask);
    int inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wcnt[w] = inc;
    __syncthreads();
    if (w == 0) {
        const int v = lane < CP_CTHREADS / 32 ? wcnt[lane] : 0;
        int wi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < CP_CTHREADS / 32) wcnt[lane] = wi - v;
        if (lane == 31) base = wi ? atomicAdd(&att->n_cand_p1, wi) : 0;
    }
    __syncthreads();
    int pos = base + wcnt[w] + inc - cnt;
    while (mask) {
        const int b = __ffs(mask) - 1;
        mask &= mask - 1;
        cand[pos] = i0 + b;
        rho_max[pos] = f2ord(-INFINITY);
        pruned[pos] = 0;
        rc_slot[pos] = -1;
        ++pos;
    }
}

// Identity list 0..C-1 of the phase-1 candidates (first refine round).
__global__ void k_list_init(const PaddiAttemptDev *att, int32_t *list, int32_t *count)
{
    const int C = att->n_cand_p1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x)
        list[i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = C;
}

// Keeps the not-yet-pruned entries of a candidate list (order within a
// block preserved), so the next refine round works on dense tiles.  out_count
// is zero on entry (every attempt starts from a zeroed PaddiAttemptDev).
__global__ void __launch_bounds__(CP_THREADS)
k_list_compact(const int32_t *__restrict__ in, const int32_t *__restrict__ in_count,
               const uint8_t *__restrict__ pruned, int32_t *out, int32_t *out_count)
{
    __shared__ int wcnt[CP_THREADS / 32];
    __shared__ int base;
    const int C = *in_count;
    for (int b0 = blockIdx.x * CP_THREADS; b0 < C; b0 += gridDim.x * CP_THREADS) {
        const int i = b0 + threadIdx.x;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const int p = i < C ? in[i] : 0;
        const bool a = i < C && !pruned[p];
        const unsigned b = __ballot_sync(0xffffffffu, a);
        if (lane == 0) wcnt[w] = __popc(b);
        __syncthreads();
        if (w == 0) {
            int v = wcnt[lane], inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            wcnt[lane] = inc - v;
            if (lane == 31) base = inc ? atomicAdd(out_count, inc) : 0;
        }
        __syncthreads();
        if (a) out[base + wcnt[w] + __popc(b & ((1u << lane) - 1u))] = p;
        __syncthreads();
    }
}

// ------------------------------------------------------------------ block helpers
template <int NT>
__device__ float block_min(float v, float *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = threadIdx.x < NT / 32 ? red[threadIdx.x] : INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = fminf(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const float r = red[0];
    __syncthreads();
    return r;
}

template <int NT>
__device__ long long block_sum(long long v, long long *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        long long t = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const long long r = red[0];
    __syncthreads();
    return r;
}

// argmax of (value, -index): larger value first, then smaller index.
struct VI {
    float v;
    int i;
};
__device__ __forceinline__ VI vi_better(VI a, VI b)
{
    if (a.v > b.v) return a;
    if (b.v > a.v) return b;
    return a.i <= b.i ? a : b;
}
template <int NT>
__device__ VI block_argmax(VI v, VI *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        VI t;
        t.v = __shfl_xor_sync(0xffffffffu, v.v, o);
        t.i = __shfl_xor_sync(0xffffffffu, v.i, o);
        v = vi_better(v, t);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        VI t = threadIdx.x < NT / 32 ? red[threadIdx.x] : VI{-INFINITY, 0x7fffffff};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            VI u;
            u.v = __shfl_xor_sync(0xffffffffu, t.v, o);
            u.i = __shfl_xor_sync(0xffffffffu, t.i, o);
            t = vi_better(t, u);
        }
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const VI r = red[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ bool overlaps(int a, int b, int m)
{
    const int d = a > b ? a - b : b - a;
    return d < m - 1;
}

// --------------------------------------------------------------- finalize
// Classifies the refined candidates and queues FP64 rechecks:
//   rho < thr - guard           -> certainly nn > r^2 (candidate and discord)
//   thr - guard <= rho <= thr+g -> borderline, exact value needed
//   and every candidate whose FP32 value could reach the top-k picks.
__global__ void __launch_bounds__(FZ_THREADS)
k_finalize(const int32_t *__restrict__ cand, PaddiAttemptDev *att,
           const uint32_t *__restrict__ rho_max, const uint8_t *__restrict__ pruned, int32_t m,
           float r2, float thr, float guard, float widen, int32_t top_k,
           const uint8_t *__restrict__ flat, int32_t rc_cap,
           int32_t *recheck, int32_t *rc_slot, unsigned long long *nn64_ord,
           PaddiAttemptResult *res, int32_t known_w, unsigned long long known_ord)
{
    __shared__ long long redl[32];
    __shared__ VI redv[32];
    __shared__ int picks[PADDI_MAX_TOPK];
    __shared__ int s_nr;
    const int C = att->n_cand_p1;
    if (threadIdx.x == 0) s_nr = 0;
    __syncthreads();
    // FP32 values far from the threshold, and flat windows (exact), are
    // classified here; the borderline ones after the recheck.
    long long certain_c = 0, certain_d = 0;
    for (int c = threadIdx.x; c < C; c += FZ_THREADS) {
        if (pruned[c]) continue;
        const float r = ord2f(rho_max[c]);
        if (flat[cand[c]]) {
            const float v = fminf(2.f * (float)m * (1.f - r), FLT_MAX);
            certain_c += v >= r2;
            certain_d += v > r2;
        } else if (r < thr - guard) {
            ++certain_c;
            ++certain_d;
        }
    }
    certain_c = block_sum<FZ_THREADS>(certain_c, redl);
    certain_d = block_sum<FZ_THREADS>(certain_d, redl);
    // FP32 greedy top-k to find the cut-off value
    int np = 0;
    float cut = INFINITY; // rho of the last pick
    for (int p = 0; p < top_k; ++p) {
        VI best{-INFINITY, 0x7fffffff};
        for (int c = threadIdx.x; c < C; c += FZ_THREADS) {
            if (pruned[c]) continue;
            const float r = ord2f(rho_max[c]);
            if (!(r <= thr + guard)) continue;
            const int w = cand[c];
            bool ex = false;
            for (int q = 0; q < np; ++q) ex |= overlaps(w, cand[picks[q]], m);
            if (ex) continue;
            best = vi_better(best, VI{-r, c});
        }
        best = block_argmax<FZ_THREADS>(best, redv);
        if (best.i == 0x7fffffff) break;
        if (threadIdx.x == 0) picks[np] = best.i;
        __syncthreads();
        ++np;
        cut = -best.v;
    }
    // queue: borderline candidates and every candidate within widen*guard of
    // the cut.  A flat window's value is exact already (rho is 0 or 1 by the
    // flat-window policy), so it is never queued.
    for (int c = threadIdx.x; c < C; c += FZ_THREADS) {
        if (pruned[c] || flat[cand[c]]) continue;
        const float r = ord2f(rho_max[c]);
        const bool border = r >= thr - guard;
        const bool neartop = np > 0 && r <= cut + widen * guard;
        if (border || neartop) {
            const int k = atomicAdd(&s_nr, 1);
            if (k < rc_cap) {
                recheck[k] = c;
                rc_slot[c] = k;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nr = s_nr;
        att->n_recheck = nr < rc_cap ? nr : rc_cap;
        att->n_recheck_all = nr;
        // a status set earlier (3: a refine wait ran out) is kept: it explains
        // an overflow here and must reach the host unchanged
        if (nr > rc_cap) atomicCAS(&att->status, 0, 1);
        res->n_p1 = C;
        res->n_recheck = nr;
        res->n_cand = certain_c; // completed in k_select
        res->n_disc = certain_d;
    }
    const int nfill = s_nr < rc_cap ? s_nr : rc_cap;
    // a window whose exact nn is already known (known_w) is filled in here and
    // skipped by the recheck
    for (int k = threadIdx.x; k < nfill; k += FZ_THREADS)
        nn64_ord[k] = (known_w >= 0 && cand[recheck[k]] == known_w) ? known_ord : d2ord(INFINITY);
}

// ---------------------------------------------------------------- recheck
// Exact FP64 nn of the queued windows.  The neighbour range is cut into
// blocks of RC_SPAN windows; a work item is (queued window, run of `per`
// consecutive blocks), with `per` chosen on the device from the queue length
// so that the items fill the grid about four times over even for one queued
// window.  Each CTA stages the centred candidate window and a slice of the
// series (FP64, shifted by its first value); each thread owns RC_JPT
// consecutive neighbour windows and slides a register ring over the slice
// (per step: one shared load of the slice, one broadcast of the candidate,
// RC_JPT FP64 FMAs).
constexpr int RC_JPT = 8;                    // neighbour windows per thread
constexpr int RC_SPAN = RC_THREADS * RC_JPT; // neighbour windows per block

__device__ __forceinline__ int rpad(int d) { return d + (d >> 4); } // conflict-free at stride 8

__global__ void __launch_bounds__(RC_THREADS)
k_recheck(const float *__restrict__ x, const double *__restrict__ mu64,
          const double *__restrict__ inv64, const uint8_t *__restrict__ flat, int32_t N,
          int32_t m, const int32_t *__restrict__ cand, const int32_t *__restrict__ recheck,
          PaddiAttemptDev *att, unsigned long long *nn64_ord, int32_t known_w)
{
    __shared__ double a[RC_MAXM];
    __shared__ double xs[RC_SPAN + RC_MAXM + (RC_SPAN + RC_MAXM) / 16 + 16];
    __shared__ double reda[RC_THREADS / 32];
    __shared__ double redm[RC_THREADS / 32];
    __shared__ int s_item;
    const int nr = att->n_recheck;
    const int nblk = (N + RC_SPAN - 1) / RC_SPAN;
    const long long want = 4ll * gridDim.x;
    const int per = (int)max(1ll, ((long long)nr * nblk) / want); // blocks per item
    const int ipc = (nblk + per - 1) / per;                        // items per queued window
    const long long total = (long long)nr * ipc;
    const int t = threadIdx.x;
    for (;;) {
        if (t == 0) s_item = atomicAdd(&att->recheck_next, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) break;
        const int r = item % nr, sp = item / nr;
        const int w = cand[recheck[r]];
        if (w == known_w) continue; // exact value filled in by the finalize step
        const double mw = mu64[w], iw = inv64[w];
        const int fw = flat[w];
        double asum = 0.0;
        for (int k = t; k < m; k += RC_THREADS) {
            const double v = (double)x[w + k] - mw;
            a[k] = v;
            asum += v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) asum += __shfl_xor_sync(0xffffffffu, asum, o);
        if ((t & 31) == 0) reda[t >> 5] = asum;
        __syncthreads();
        asum = 0.0;
        for (int q = 0; q < RC_THREADS / 32; ++q) asum += reda[q];
        double best = INFINITY;
        const int j_lo = sp * per * RC_SPAN;
        const int j_hi = (int)min((long long)N, (long long)j_lo + (long long)per * RC_SPAN);
        for (int j0 = j_lo; j0 < j_hi; j0 += RC_SPAN) {
            __syncthreads();
            const double sh = (double)x[j0];
            for (int p = t; p < RC_SPAN + m + RC_JPT; p += RC_THREADS) {
                const int g = j0 + p;
                xs[rpad(p)] = (g < N + m - 1 ? (double)x[g] : sh) - sh;
            }
            __syncthreads();
            const int q0 = RC_JPT * t;
            double acc[RC_JPT], ring[RC_JPT];
#pragma unroll
            for (int c = 0; c < RC_JPT; ++c) {
                acc[c] = 0.0;
                ring[c] = xs[rpad(q0 + c)];
            }
            for (int k0 = 0; k0 < m; k0 += RC_JPT) {
#pragma unroll
                for (int u = 0; u < RC_JPT; ++u) {
                    if (k0 + u < m) {
                        const double ak = a[k0 + u];
#pragma unroll
                        for (int c = 0; c < RC_JPT; ++c)
                            acc[c] = fma(ak, ring[(u + c) & (RC_JPT - 1)], acc[c]);
                    }
                    ring[u] = xs[rpad(q0 + k0 + u + RC_JPT)];
                }
            }
#pragma unroll
            for (int c = 0; c < RC_JPT; ++c) {
                const int j = j0 + q0 + c;
                if (j < j_hi && !overlaps(w, j, m)) {
                    const double cov = acc[c] - (mu64[j] - sh) * asum;
                    double rho;
                    if (fw | flat[j]) rho = (fw & flat[j]) ? 1.0 : 0.0;
                    else rho = cov * iw * inv64[j];
                    double d = 2.0 * m * (1.0 - rho);
                    d = d < 0.0 ? 0.0 : d;
                    best = fmin(best, d);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, o));
        if ((t & 31) == 0) redm[t >> 5] = best;
        __syncthreads();
        if (t == 0) {
            double b = INFINITY;
            for (int q = 0; q < RC_THREADS / 32; ++q) b = fmin(b, redm[q]);
            atomicMin(nn64_ord + r, d2ord(b));
        }
    }
}

// ----------------------------------------------------------------- select
// Final counts and greedy top-k with exact values where they matter.
// status 2: a pick has no exact value yet (host appends it and re-runs).
__global__ void __launch_bounds__(FZ_THREADS)
k_select(const int32_t *__restrict__ cand, PaddiAttemptDev *att,
         const uint32_t *__restrict__ rho_max, const uint8_t *__restrict__ pruned,
         const int32_t *__restrict__ recheck, const int32_t *__restrict__ rc_slot,
         const unsigned long long *__restrict__ nn64_ord, int32_t m, float r2, float thr,
         float guard, int32_t top_k, const uint8_t *__restrict__ flat, PaddiAttemptResult *res)
{
    __shared__ long long redl[32];
    __shared__ VI redv[32];
    __shared__ int picks_w[PADDI_MAX_TOPK];
    __shared__ int s_need;
    const int C = att->n_cand_p1;
    const int nr = att->n_recheck;
    if (threadIdx.x == 0) s_need = 0;
    __syncthreads();
    // exact classification of the rechecked borderline windows
    long long addc = 0, addd = 0;
    for (int k = threadIdx.x; k < nr; k += FZ_THREADS) {
        const int c = recheck[k];
        const float r = ord2f(rho_max[c]);
        if (r >= thr - guard && !flat[cand[c]]) { // borderline (certain ones were already counted)
            const float v = (float)fmin(ord2d(nn64_ord[k]), (double)FLT_MAX);
            addc += v >= r2;
            addd += v > r2;
        }
    }
    addc = block_sum<FZ_THREADS>(addc, redl);
    addd = block_sum<FZ_THREADS>(addd, redl);
    // greedy top-k among nn > r2
    int np = 0;
    for (int p = 0; p < top_k; ++p) {
        VI best{-INFINITY, 0x7fffffff};
        for (int c = threadIdx.x; c < C; c += FZ_THREADS) {
            if (pruned[c]) continue;
            const float r = ord2f(rho_max[c]);
            if (!(r <= thr + guard)) continue;
            // exact value if rechecked, else the FP32 estimate
            float v = (float)fmin((double)(2.f * m * (1.f - r)), (double)FLT_MAX);
            const int slot = rc_slot[c];
            if (slot >= 0) v = (float)fmin(ord2d(nn64_ord[slot]), (double)FLT_MAX);
            else if (r >= thr - guard && !flat[cand[c]]) continue; // no exact value (overflow)
            if (!(v > r2)) continue;
            const int w = cand[c];
            bool ex = false;
            for (int q = 0; q < np; ++q) ex |= overlaps(w, picks_w[q], m);
            if (ex) continue;
            best = vi_better(best, VI{v, w});
        }
        best = block_argmax<FZ_THREADS>(best, redv);
        if (best.i == 0x7fffffff) break;
        if (threadIdx.x == 0) {
            picks_w[np] = best.i;
            res->sel_ind[np] = best.i;
            res->sel_dist[np] = best.v;
        }
        __syncthreads();
        ++np;
    }
    // every pick must carry an exact value
    for (int q = 0; q < np; ++q) {
        const int wq = picks_w[q];
        bool found = flat[wq] != 0;
        for (int k = threadIdx.x; k < nr; k += FZ_THREADS) found |= cand[recheck[k]] == wq;
        found = __syncthreads_or(found);
        if (!found && threadIdx.x == 0) s_need = 1;
    }
    (void)recheck;
    __syncthreads();
    if (threadIdx.x == 0) {
        res->n_cand += addc;
        res->n_disc += addd;
        res->n_sel = np;
        // the full count, so the host can size the queue after an overflow
        res->n_recheck = att->n_recheck_all;
        res->n_pairs = att->n_pairs;
        res->n_live = att->n_live;
        res->p1_walked = att->p1_walked;
        res->status = att->status ? att->status : (s_need ? 2 : 0);
    }
}

// Candidate flags and distances in the reference's per-window layout
// (d_is_cand / d_nnDist of do_PD3, src/PD3.cuh:15).
__global__ void k_scatter_clear(int32_t N, int32_t *is_cand, float *nnd)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    is_cand[i] = 0;
    nnd[i] = -FLT_MAX;
}

__global__ void k_scatter(const int32_t *__restrict__ cand, const PaddiAttemptDev *att,
                          const uint32_t *__restrict__ rho_max, const uint8_t *__restrict__ pruned,
                          const int32_t *__restrict__ rc_slot,
                          const unsigned long long *__restrict__ nn64_ord,
                          const uint8_t *__restrict__ flat, int32_t m, float r2, int32_t *is_cand,
                          float *nnd)
{
    const int C = att->n_cand_p1;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        if (pruned[c]) continue;
        const int w = cand[c];
        const int slot = rc_slot[c];
        float v;
        if (slot >= 0) v = (float)fmin(ord2d(nn64_ord[slot]), (double)FLT_MAX);
        else v = fminf(2.f * (float)m * (1.f - ord2f(rho_max[c])), FLT_MAX);
        if (v >= r2) {
            is_cand[w] = 1;
            nnd[w] = v;
        }
    }
}

} // namespace

cudaError_t paddi_launch_list_init(const PaddiAttemptDev *att, int32_t *list, int32_t *count,
                                   cudaStream_t st)
{
    k_list_init<<<256, 256, 0, st>>>(att, list, count);
    return cudaGetLastError();
}

cudaError_t paddi_launch_list_compact(const int32_t *in, const int32_t *in_count,
                                      const uint8_t *pruned, int32_t *out, int32_t *out_count,
                                      cudaStream_t st)
{
    k_list_compact<<<64, CP_THREADS, 0, st>>>(in, in_count, pruned, out, out_count);
    return cudaGetLastError();
}

cudaError_t paddi_launch_scatter(const int32_t *cand, const PaddiAttemptDev *att,
                                 const uint32_t *rho_max, const uint8_t *pruned,
                                 const int32_t *rc_slot, const unsigned long long *nn64_ord,
                                 const uint8_t *flat, int32_t N, int32_t m, float r2,
                                 int32_t *is_cand, float *nnd, cudaStream_t st)
{
    k_scatter_clear<<<(N + 255) / 256, 256, 0, st>>>(N, is_cand, nnd);
    k_scatter<<<256, 256, 0, st>>>(cand, att, rho_max, pruned, rc_slot, nn64_ord, flat, m, r2,
                                   is_cand, nnd);
    return cudaGetLastError();
}

cudaError_t paddi_launch_compact(const uint8_t *alive, int32_t N, int32_t *cand,
                                 uint32_t *rho_max, uint8_t *pruned, int32_t *rc_slot,
                                 PaddiAttemptDev *att, const uint8_t *flat,
                                 const int32_t *flat_span, int32_t m, bool prune_flats,
                                 cudaStream_t st)
{
    const int per_cta = CP_CTHREADS * CP_WIN;
    const unsigned grid = (unsigned)((N + per_cta - 1) / per_cta);
    k_compact<<<grid, CP_CTHREADS, 0, st>>>(alive, N, cand, rho_max, pruned, rc_slot, att, flat,
                                           flat_span, m, prune_flats ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t paddi_launch_finalize(const int32_t *cand, PaddiAttemptDev *att,
                                  const uint32_t *rho_max, const uint8_t *pruned, int32_t m,
                                  float r2, float thr, float guard, float widen, int32_t top_k,
                                  const uint8_t *flat, int32_t rc_cap, int32_t *recheck,
                                  int32_t *rc_slot, unsigned long long *nn64_ord,
                                  PaddiAttemptResult *res, int32_t known_w,
                                  unsigned long long known_ord, cudaStream_t st)
{
    if (top_k < 1 || top_k > PADDI_MAX_TOPK) return cudaErrorInvalidValue;
    k_finalize<<<1, FZ_THREADS, 0, st>>>(cand, att, rho_max, pruned, m, r2, thr, guard, widen,
                                         top_k, flat, rc_cap, recheck, rc_slot, nn64_ord, res,
                                         known_w, known_ord);
    return cudaGetLastError();
}

cudaError_t paddi_launch_recheck(const float *x, const double *mu64, const double *inv64,
                                 const uint8_t *flat, int32_t N, int32_t m,
                                 const int32_t *cand, const int32_t *recheck,
                                 PaddiAttemptDev *att, unsigned long long *nn64_ord,
                                 int32_t num_sms, int32_t known_w, cudaStream_t st)
{
    if (m > RC_MAXM) return cudaErrorInvalidValue;
    k_recheck<<<num_sms * 4, RC_THREADS, 0, st>>>(x, mu64, inv64, flat, N, m, cand, recheck, att,
                                                 nn64_ord, known_w);
    return cudaGetLastError();
}

cudaError_t paddi_launch_select(const int32_t *cand, PaddiAttemptDev *att,
                                const uint32_t *rho_max, const uint8_t *pruned,
                                const int32_t *recheck, const int32_t *rc_slot,
                                const unsigned long long *nn64_ord, int32_t m, float r2,
                                float thr, float guard, int32_t top_k, const uint8_t *flat,
                                PaddiAttemptResult *res, cudaStream_t st)
{
    k_select<<<1, FZ_THREADS, 0, st>>>(cand, att, rho_max, pruned, recheck, rc_slot, nn64_ord,
                                       m, r2, thr, guard, top_k, flat, res);
    return cudaGetLastError();
}
