// k_phase1.cu -- phase 1 of PD3: candidate selection by diagonal strips.
//
// Reference: gpu_local_candidate_select (src/PD3_kernels.cuh:9-259).  Each
// reference block owns SEGMENT_N windows ("rows"), walks 512-window chunks to
// the right with a diagonal dot-product recurrence (one __syncthreads per
// diagonal step), prunes a row as soon as one admissible neighbour is closer
// than r, marks that neighbour too (atomicMin(d_neighbor+j, 0), :74-78), and
// leaves once every row of the block is pruned (:130-146).
//
// B200 form:
//   * a persistent grid pulls (segment, chunk) tasks chunk-major from a
//     global counter, so every segment's nearest chunk is done before any
//     segment continues, and segments whose rows are all pruned drop out;
//   * a task is R rows x 256 diagonals, walked by one warp; each lane owns
//     the 4 diagonals 4t..4t+3 and their partners 128 further on, and walks
//     all R rows with the centred covariance update
//         cov(i+1, j+1) = cov(i, j) + df_i dg_j + df_j dg_i
//     on (diagonal, partner) pairs with packed f32x2 FMAs; the column
//     operands come pair-packed from shared memory ((col q, col q+128) per
//     entry, XOR-swizzled so the stride-4 ring loads are conflict-free) and
//     rotate through a 4-entry register ring, one entry per row step.  Short
//     chunks let most segments stop early: after the first 256 diagonals
//     nearly every row of most segments is pruned;
//   * the starting covariances of the 256 diagonals are m-term dot products
//     of the centred first row window with the shifted series;
//   * hits are tracked as running maxima of rho (per row step over the
//     thread's 8 diagonals; per column over the rows that touch it), and only
//     the maxima are compared with the threshold: a row is pruned through one
//     warp ballot per step, a column when it leaves the thread's ring; both
//     go to shared-memory byte flags and are flushed as byte stores of 0 to
//     the global alive[] array (idempotent, so no atomics).
// Pruning uses rho > thr_prune where thr_prune = 1 - r^2/(2m) + guard, so a
// window is pruned only when its FP32 correlation clears the threshold by
// more than the rounding bound; everything else stays a candidate and is
// settled by the refine and the FP64 recheck.
// A flat window has inv = 0, so every pair with one gets rho = 0 here.  That
// is exact against a non-flat window (the reference's d = 2m) and low for a
// flat-flat pair (exactly rho = 1): such pairs prune nothing in this pass.
// The candidate compaction drops flat windows with an admissible flat partner
// instead, from the span of the flat windows (exact: their distance is 0).
#include <algorithm>

#include "paddi_internal.cuh"

namespace {

constexpr int P1_THREADS = 32;                // one warp per task
constexpr int P1_GPT = 4;                     // diagonal pairs per thread
constexpr int P1_H = P1_THREADS * P1_GPT;     // partner offset (128)
constexpr int P1_D = 2 * P1_H;                // diagonals per chunk
constexpr int P1_MAXM = 1024;

// pair-packed column arrays: stride-4 float4 / float2 loads conflict-free
__host__ __device__ __forceinline__ int csw(int q) { return q ^ ((q >> 2) & 15); }
__host__ __device__ __forceinline__ int xpad(int p) { return p + (p >> 5); } // stride-4 floats
__host__ __device__ __forceinline__ int p1_ncp(int R) { return (R + P1_H + 63) & ~63; }

// max(a, b, c) in one instruction (sm_100 three-input form)
__device__ __forceinline__ float fmax3(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

struct P1Smem {
    float4 *roww;     // R
    float2 *colz;     // ncp: (inv_q, inv_q+H)
    float4 *colxy;    // ncp: (df_q, df_q+H, dg_q, dg_q+H); aliases xa / xb
    float *xa;        // mpad
    float *xb;        // xpad(D + mpad + 8)
    uint8_t *colflag; // R + D
    uint8_t *rowflag; // R
};

template <bool BOUND>
__device__ __forceinline__ void p1_walk(const P1Smem &S, float2 (&cov)[P1_GPT], int R, int rows,
                                        int lim, float thr, int t)
{
    const int lane = threadIdx.x & 31;
    const int c0 = P1_GPT * t;
    float4 rxy[4];
    float2 rz[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        rxy[k] = S.colxy[csw(c0 + k)];
        rz[k] = S.colz[csw(c0 + k)];
    }
    float cmA[4], cmB[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) cmA[k] = cmB[k] = -INFINITY;
    for (int s0 = 0; s0 < R; s0 += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int s = s0 + u;
            const float4 ri = S.roww[s];
            const float2 rix = make_float2(ri.x, ri.x), riy = make_float2(ri.y, ri.y);
            const float2 riz = make_float2(ri.z, ri.z);
            float rmax = -INFINITY;
#pragma unroll
            for (int k = 0; k < P1_GPT; ++k) {
                const int sl = (u + k) & 3;
                const float2 cx = make_float2(rxy[sl].x, rxy[sl].y);
                const float2 cy = make_float2(rxy[sl].z, rxy[sl].w);
                float2 rho = __fmul2_rn(__fmul2_rn(cov[k], riz), rz[sl]);
                if (BOUND) {
                    const int q = s + c0 + k;
                    if (s >= rows || q >= lim) rho.x = -INFINITY;
                    if (s >= rows || q + P1_H >= lim) rho.y = -INFINITY;
                }
                rmax = fmax3(rmax, rho.x, rho.y);
                cmA[sl] = fmaxf(cmA[sl], rho.x);
                cmB[sl] = fmaxf(cmB[sl], rho.y);
                cov[k] = __ffma2_rn(rix, cy, __ffma2_rn(cx, riy, cov[k]));
            }
            if (__ballot_sync(0xffffffffu, rmax > thr) && lane == 0) S.rowflag[s] = 1;
            // columns s + c0 and s + c0 + H leave the ring: no later row touches them
            if (cmA[u] > thr) S.colflag[s + c0] = 1;
            if (cmB[u] > thr) S.colflag[s + c0 + P1_H] = 1;
            cmA[u] = -INFINITY;
            cmB[u] = -INFINITY;
            const int qn = csw(s + c0 + 4);
            rxy[u] = S.colxy[qn];
            rz[u] = S.colz[qn];
        }
    }
    // columns R + c0 + e (e < 3) were touched by the last rows only
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        if (cmA[e] > thr) S.colflag[R + c0 + e] = 1;
        if (cmB[e] > thr) S.colflag[R + c0 + e + P1_H] = 1;
    }
}

__global__ void __launch_bounds__(P1_THREADS, 16)
k_phase1(const float *__restrict__ x, const float4 *__restrict__ wst, const float *__restrict__ mu,
         uint8_t *alive, int32_t N, int32_t m, int32_t R, int32_t max_chunks, float thr,
         int32_t *task_counter, int32_t *walked)
{
    extern __shared__ __align__(16) unsigned char p1_smem[];
    const int mpad = (m + 7) & ~7;
    const int ncp = p1_ncp(R);
    P1Smem S;
    S.roww = reinterpret_cast<float4 *>(p1_smem);
    S.colz = reinterpret_cast<float2 *>(S.roww + R);
    S.colxy = reinterpret_cast<float4 *>(S.colz + ncp);
    S.xa = reinterpret_cast<float *>(S.colxy);
    S.xb = S.xa + mpad;
    const size_t ubytes = max((size_t)16 * ncp,
                              (size_t)4 * (mpad + xpad(P1_D + mpad + 8) + 1));
    S.colflag = reinterpret_cast<uint8_t *>(S.colxy) + ((ubytes + 15) & ~(size_t)15);
    S.rowflag = S.colflag + R + P1_D;
    __shared__ int s_task;
    __shared__ float s_red[P1_THREADS / 32];

    const int t = threadIdx.x;
    const int c0 = P1_GPT * t;
    const int nseg = (N + R - 1) / R;
    const int total = nseg * max_chunks;
    for (;;) {
        if (t == 0) s_task = atomicAdd(task_counter, 1);
        __syncthreads();
        const int task = s_task;
        if (task >= total) break;
        const int chunk = task / nseg, seg = task - chunk * nseg;
        const int i0 = seg * R;
        const int rows = min(R, N - i0);
        const int d0 = (m - 1) + chunk * P1_D;
        if (i0 + d0 >= N) { // no admissible pair in this task
            __syncthreads();
            continue;
        }
        if (chunk > 0) { // continue only while some row is still a candidate
            int any = 0;
            for (int s = t; s < rows; s += P1_THREADS) any |= __ldcg(alive + i0 + s);
            any = __syncthreads_or(any);
            if (!any) continue;
        }
        // ---- stage rows, flags, the inv column pairs and the series
        //      slices for the start dots
        for (int s = t; s < R; s += P1_THREADS) {
            S.roww[s] = wst[i0 + s]; // zero beyond N (padded tail)
            S.rowflag[s] = 0;
        }
        const int cbase = i0 + d0;
        for (int q = t; q < R + P1_D; q += P1_THREADS) S.colflag[q] = 0;
        for (int q = t; q < R + P1_H; q += P1_THREADS) {
            const float4 a = wst[cbase + q], b = wst[cbase + q + P1_H];
            S.colz[csw(q)] = make_float2(a.z, b.z);
        }
        const float mu0 = mu[i0];
        float zs = 0.f;
        for (int q = t; q < mpad; q += P1_THREADS) {
            const float v = q < m ? x[i0 + q] - mu0 : 0.f;
            S.xa[q] = v;
            zs += v;
        }
        const float shift = mu[cbase];
        const int64_t nser = (int64_t)N + m - 1;
        for (int p = t; p < P1_D + mpad + 8; p += P1_THREADS) {
            const int64_t g = (int64_t)cbase + p;
            S.xb[xpad(p)] = (g < nser ? x[g] : x[nser - 1]) - shift;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) zs += __shfl_xor_sync(0xffffffffu, zs, o);
        if ((t & 31) == 0) s_red[t >> 5] = zs;
        __syncthreads();
        float zsum = 0.f;
#pragma unroll
        for (int w = 0; w < P1_THREADS / 32; ++w) zsum += s_red[w];

        // ---- starting covariances of diagonals d0 + c0 + k and d0 + c0 + k + H
        float2 cov[P1_GPT];
        {
            // (diagonal, partner) pairs with packed f32x2 FMAs: bb[i] holds the
            // series values of both diagonals of a ring slot
            float2 acc[P1_GPT], bb[4];
#pragma unroll
            for (int k = 0; k < P1_GPT; ++k) {
                acc[k] = make_float2(0.f, 0.f);
                bb[k] = make_float2(S.xb[xpad(c0 + k)], S.xb[xpad(c0 + P1_H + k)]);
            }
            for (int q0 = 0; q0 < mpad; q0 += 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float a = S.xa[q0 + u];
                    const float2 a2 = make_float2(a, a);
#pragma unroll
                    for (int k = 0; k < P1_GPT; ++k) acc[k] = __ffma2_rn(a2, bb[(u + k) & 3], acc[k]);
                    bb[u] = make_float2(S.xb[xpad(c0 + q0 + u + 4)], S.xb[xpad(c0 + P1_H + q0 + u + 4)]);
                }
            }
#pragma unroll
            for (int k = 0; k < P1_GPT; ++k) {
                const int ja = cbase + c0 + k, jb = ja + P1_H;
                const float mua = ja < N ? mu[ja] : shift;
                const float mub = jb < N ? mu[jb] : shift;
                cov[k] = make_float2(fmaf(-(mua - shift), zsum, acc[k].x),
                                     fmaf(-(mub - shift), zsum, acc[k].y));
            }
        }
        __syncthreads(); // xa / xb are overwritten by the (df, dg) column pairs
        for (int q = t; q < R + P1_H; q += P1_THREADS) {
            const float4 a = wst[cbase + q], b = wst[cbase + q + P1_H];
            S.colxy[csw(q)] = make_float4(a.x, b.x, a.y, b.y);
        }
        __syncthreads();
        // ---- walk the R rows
        if (t == 0) atomicAdd(walked, 1);
        const int lim = N - cbase; // column q is a window iff q < lim
        const bool bound = (rows < R) || (R + P1_D > lim);
        if (bound && thr < 0.f) p1_walk<true>(S, cov, R, rows, lim, thr, t);
        else p1_walk<false>(S, cov, R, rows, lim, thr, t);
        __syncthreads();
        // ---- flush pruning marks
        for (int s = t; s < rows; s += P1_THREADS)
            if (S.rowflag[s]) alive[i0 + s] = 0;
        for (int q = t; q < R + P1_D; q += P1_THREADS)
            if (S.colflag[q] && q < lim) alive[cbase + q] = 0;
        __syncthreads();
    }
}

} // namespace

size_t paddi_phase1_smem(int R, int m)
{
    const int mpad = (m + 7) & ~7;
    const int ncp = p1_ncp(R);
    size_t b = sizeof(float4) * (size_t)R;                  // roww
    b += sizeof(float2) * (size_t)ncp;       // colz
    const size_t ubytes = std::max((size_t)16 * ncp,
                                   (size_t)4 * (mpad + xpad(P1_D + mpad + 8) + 1));
    b += (ubytes + 15) & ~(size_t)15;        // colxy / xa + xb
    b += (size_t)(R + P1_D) + (size_t)R;     // flags
    return (b + 15) & ~(size_t)15;
}

cudaError_t paddi_launch_phase1_dev(const float *x, const float4 *wst, const float *mu,
                                    uint8_t *alive, int32_t N, int32_t m, int32_t R,
                                    int32_t max_chunks, float thr_prune,
                                    int32_t *task_counter, int32_t *walked, int32_t num_sms,
                                    cudaStream_t st)
{
    if (R < 64 || R > 4096 || (R & 7) || m > P1_MAXM || max_chunks < 1)
        return cudaErrorInvalidValue;
    const size_t smem = paddi_phase1_smem(R, m);
    cudaError_t e = paddi_raise_smem_limit((const void *)k_phase1, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase1, P1_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int nseg = (N + R - 1) / R;
    int grid = num_sms * per_sm;
    if (grid > nseg * max_chunks) grid = nseg * max_chunks;
    k_phase1<<<grid, P1_THREADS, smem, st>>>(x, wst, mu, alive, N, m, R, max_chunks, thr_prune,
                                             task_counter, walked);
    return cudaGetLastError();
}
