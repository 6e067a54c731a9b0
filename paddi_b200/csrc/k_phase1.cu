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
//     rotate through a 4-entry register ring, one entry per row step;
//   * the pair test is done in covariance units:
//         d(i, j) < r^2  <=>  rho > thr  <=>  v = cov * inv_j - thr * n_i > 0
//     (n_i = |x_i - mu_i|, inv_j = 1 / n_j), one packed FMA per pair; v > 0
//     prunes the row and the column alike, so one value feeds both the row's
//     maximum (one warp ballot per row) and the column's (merged over two
//     rows with three-input maxima, compared when the column leaves the ring);
//     prune marks go to shared-memory byte flags and are flushed as byte
//     stores of 0 to the global alive[] array (idempotent, no atomics);
//   * the starting covariances of the 256 diagonals are m-term dot products
//     of the centred first row window with the shifted series, summed in
//     blocks of 64 terms.
//
// Soundness.  A row or column is pruned only when the exact correlation is
// above thr: the FP32 rounding of the whole computation is bounded per task
// and subtracted from the covariances before the walk, so no per-pair guard
// is needed (u = 2^-24; norms come from wst[].w, FP32, widened by 2u):
//   * start dot products (row window a, centred with a two-float FP64 mean;
//     column window b shifted by s): |err| <= n_i0 ((2 g + 8u) |b_j - s| +
//     2 g_z u sqrt(m) |mu_j|) with |b_j - s| <= n_j + sqrt(m) |mu_j - s|,
//     g = (64 + ceil(m/64) + 2) u for the blocked sums and g_z = (m/32 + 6) u
//     for the row window's sum (which should be 0);
//   * one step of the recurrence (two FMAs on FP32-rounded update terms):
//     |err| <= u (2 n_i n_j + 4 (|df_j dg_i| + |df_i dg_j|)), bounded with the
//     maxima N_r, N_c, F_r, G_r, F_c, G_c of the task's rows and columns;
//     32 steps' worth is subtracted at the start of every 32-row block;
//   * the test itself (FP32 inv_j, T_i = thr n_i rounded once): 4u N_r N_c;
//   * every subtraction's own rounding: 2u N_r N_c.
// The sum is scaled by 1.01 for second-order terms.
// A flat window (all m values equal, inv = 0, n = 0) has rho = 0 against any
// other window by the flat-window rule: its row threshold T is +inf when
// thr >= 0 (no prune: 0 > thr is false) and -inf when thr < 0 (prune: d = 2m
// < r^2), and as a column it contributes v = -T_i.  Flat-flat pairs (d = 0)
// are settled at candidate compaction instead, from the span of the flat windows.
#include <algorithm>
#include <float.h>

#include "paddi_internal.cuh"

namespace {

constexpr int P1_THREADS = 32;                // one warp per task
constexpr int P1_GPT = 4;                     // diagonal pairs per thread
constexpr int P1_H = P1_THREADS * P1_GPT;     // partner offset (128)
constexpr int P1_D = 2 * P1_H;                // diagonals per chunk
static_assert(P1_GPT == 4, "the walk's ring and row maximum are written for 4 pairs");
constexpr int P1_MAXM = 1024;
constexpr int P1_SUMBLK = 64;                 // start dot products: terms per partial sum
constexpr float kU = 5.9604645e-8f;           // unit roundoff of FP32 (2^-24)

// pair-packed column arrays: stride-4 float4 / float2 loads conflict-free
__host__ __device__ __forceinline__ int csw(int q) { return q ^ ((q >> 2) & 15); }
// start-dot series pairs (float2 at stride 4 entries): one pad entry per 16
__host__ __device__ __forceinline__ int bpad(int p) { return p + (p >> 4); }
__host__ __device__ __forceinline__ int p1_ncp(int R) { return (R + P1_H + 63) & ~63; }
__host__ __device__ __forceinline__ int p1_nbp(int m) { return bpad(P1_H + ((m + 7) & ~7) + 8); }

// max(a, b, c) in one instruction (sm_100 three-input form)
__device__ __forceinline__ float fmax3(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// an FP32 norm from wst[].w (0 for flat / padded windows) rounded up to a bound
__device__ __forceinline__ float norm_up(float n) { return n * (1.f + 2.f * kU); }

struct P1Smem {
    float4 *rowdg;    // R: {df, dg, -T, 0} of the row, T = thr * n_i (one entry: more
                      // tasks fit an SM's shared memory; the packed pairs are built
                      // in registers)
    float2 *colz;     // ncp: (inv_q, inv_q+H)
    float4 *colxy;    // ncp: (df_q, df_q+H, dg_q, dg_q+H)
    float2 *xa2;      // mpad: (a_q, a_q), the centred first row window (start dots)
    float2 *xb2;      // bpad(H + mpad + 8): (y_p, y_p+H), the shifted series (start dots)
    uint8_t *colflag; // R + D
    uint8_t *rowflag; // R
};

// Walks rows [0, R) of the task.  cov holds the covariances of the lane's
// diagonals at row 0, already lowered by the start and comparison margins;
// dsub (the next 32 steps' rounding bound) is subtracted at the start of
// every 32-row block.
template <bool BOUND>
__device__ __forceinline__ void p1_walk(const P1Smem &S, float2 (&cov)[P1_GPT], int R, int rows,
                                        int lim, float dsub, int t)
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
    // column maxima per ring slot: x = column q, y = column q + H
    float2 cm[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) cm[k] = make_float2(-INFINITY, -INFINITY);
    const float2 dsub2 = make_float2(-dsub, -dsub);

    // one row: v[k] for the 4 diagonal pairs, the row's ballot, the update
    auto row = [&](int s, int u, float2 (&v)[P1_GPT]) {
        const float4 rd = S.rowdg[s];
        const float2 rt = make_float2(rd.z, rd.z);
        const float2 rix = make_float2(rd.x, rd.x), riy = make_float2(rd.y, rd.y);
#pragma unroll
        for (int k = 0; k < P1_GPT; ++k) {
            const int sl = (u + k) & 3;
            float2 vv = __ffma2_rn(cov[k], rz[sl], rt);
            if (BOUND) {
                const int q = s + c0 + k;
                if (s >= rows || q >= lim) vv.x = -INFINITY;
                if (s >= rows || q + P1_H >= lim) vv.y = -INFINITY;
            }
            v[k] = vv;
            const float2 cx = make_float2(rxy[sl].x, rxy[sl].y);
            const float2 cy = make_float2(rxy[sl].z, rxy[sl].w);
            cov[k] = __ffma2_rn(rix, cy, __ffma2_rn(cx, riy, cov[k]));
        }
        // the row's maximum as a tree of depth 2, off the walk's dependency chain
        const float rmax = fmax3(fmax3(v[0].x, v[0].y, v[1].x), fmax3(v[1].y, v[2].x, v[2].y),
                                 fmaxf(v[3].x, v[3].y));
        if (__ballot_sync(0xffffffffu, rmax > 0.f) && lane == 0) S.rowflag[s] = 1;
    };
    // the column in ring slot sl leaves: flag it, load column q + 4 into the slot
    auto leave = [&](int sl, int q) {
        if (cm[sl].x > 0.f) S.colflag[q] = 1;
        if (cm[sl].y > 0.f) S.colflag[q + P1_H] = 1;
        cm[sl] = make_float2(-INFINITY, -INFINITY);
        const int qn = csw(q + 4);
        rxy[sl] = S.colxy[qn];
        rz[sl] = S.colz[qn];
    };

    for (int s0 = 0; s0 < R; s0 += 4) {
        if ((s0 & 31) == 0) {
#pragma unroll
            for (int k = 0; k < P1_GPT; ++k) cov[k] = __fadd2_rn(cov[k], dsub2);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            // rows s (ring offset u) and s + 1 (u + 1); at row s diagonal k
            // meets the column in slot (u + k) & 3, at row s + 1 slot (u + 1 + k) & 3
            const int u = 2 * h, s = s0 + u;
            float2 v0[P1_GPT], v1[P1_GPT];
            row(s, u, v0);
            cm[u].x = fmaxf(cm[u].x, v0[0].x); // column c0 + s: last touched by row s
            cm[u].y = fmaxf(cm[u].y, v0[0].y);
            leave(u, s + c0);
            row(s + 1, u + 1, v1);
            const int s1 = (u + 1) & 3, s2 = (u + 2) & 3, s3 = (u + 3) & 3;
            cm[s1].x = fmax3(cm[s1].x, v0[1].x, v1[0].x);
            cm[s1].y = fmax3(cm[s1].y, v0[1].y, v1[0].y);
            leave(s1, s + 1 + c0);
            cm[s2].x = fmax3(cm[s2].x, v0[2].x, v1[1].x);
            cm[s2].y = fmax3(cm[s2].y, v0[2].y, v1[1].y);
            cm[s3].x = fmax3(cm[s3].x, v0[3].x, v1[2].x);
            cm[s3].y = fmax3(cm[s3].y, v0[3].y, v1[2].y);
            cm[u] = v1[3]; // column c0 + s + 4, loaded after row s
        }
    }
    // columns R + c0 + e (e < 3) were touched by the last rows only
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const int sl = (R + e) & 3;
        if (cm[sl].x > 0.f) S.colflag[R + c0 + e] = 1;
        if (cm[sl].y > 0.f) S.colflag[R + c0 + e + P1_H] = 1;
    }
}

__global__ void __launch_bounds__(P1_THREADS, 16)
k_phase1(const float *__restrict__ x, const float4 *__restrict__ wst, const float *__restrict__ mu,
         const double *__restrict__ mu64, uint8_t *alive, int32_t N, int32_t m, int32_t R,
         int32_t max_chunks, float thr, int32_t row_lo, int32_t row_hi, int32_t *task_counter,
         int32_t *walked)
{
    extern __shared__ __align__(16) unsigned char p1_smem[];
    const int mpad = (m + 7) & ~7;
    const int ncp = p1_ncp(R);
    P1Smem S;
    S.rowdg = reinterpret_cast<float4 *>(p1_smem);
    S.colxy = reinterpret_cast<float4 *>(S.rowdg + R);
    S.colz = reinterpret_cast<float2 *>(S.colxy + ncp);
    S.xa2 = reinterpret_cast<float2 *>(S.colxy); // start dots: aliases the column arrays
    S.xb2 = S.xa2 + mpad;
    const size_t ubytes = max((size_t)24 * ncp, (size_t)8 * (mpad + p1_nbp(m)));
    S.colflag = reinterpret_cast<uint8_t *>(S.colxy) + ((ubytes + 15) & ~(size_t)15);
    S.rowflag = S.colflag + R + P1_D;
    __shared__ int s_task;

    const int t = threadIdx.x;
    const int c0 = P1_GPT * t;
    const int nseg = (row_hi - row_lo + R - 1) / R; // segments of the row range
    const int total = nseg * max_chunks;
    const float sqrtm = sqrtf((float)m) * (1.f + 2.f * kU);
    // rounding-bound constants of the start dot products
    const float g_dot = (float)(P1_SUMBLK + (mpad + P1_SUMBLK - 1) / P1_SUMBLK + 2) * kU;
    const float g_z = (float)(mpad / 32 + 6) * kU;
    for (;;) {
        if (t == 0) s_task = atomicAdd(task_counter, 1);
        __syncwarp();
        const int task = s_task;
        __syncwarp();
        if (task >= total) break;
        const int chunk = task / nseg, seg = task - chunk * nseg;
        const int i0 = row_lo + seg * R;
        const int rows = min(R, row_hi - i0);
        const int d0 = (m - 1) + chunk * P1_D;
        if (i0 + d0 >= N) continue; // no admissible pair in this task
        if (chunk > 0) { // continue only while some row is still a candidate
            int any = 0;
            for (int s = t; s < rows; s += P1_THREADS) any |= __ldcg(alive + i0 + s);
            if (!__any_sync(0xffffffffu, any)) continue;
        }
        // ---- rows: update terms, thresholds T_i = thr n_i, flags, maxima
        float nr = 0.f, fr = 0.f, gr = 0.f;
        for (int s = t; s < R; s += P1_THREADS) {
            const float4 w = wst[i0 + s]; // zero beyond N (padded tail)
            const float T = w.z > 0.f ? thr * w.w : (thr < 0.f ? -INFINITY : INFINITY);
            S.rowdg[s] = make_float4(w.x, w.y, -T, 0.f);
            S.rowflag[s] = 0;
            nr = fmaxf(nr, w.w);
            fr = fmaxf(fr, fabsf(w.x));
            gr = fmaxf(gr, fabsf(w.y));
        }
        const int cbase = i0 + d0;
        for (int q = t; q < R + P1_D; q += P1_THREADS) S.colflag[q] = 0;
        // ---- start dot products: row window centred with its two-float mean,
        //      series shifted by the first column window's mean
        const double m0 = mu64[i0];
        const float mhi = (float)m0, mlo = (float)(m0 - (double)mhi);
        float zs = 0.f;
        for (int q = t; q < mpad; q += P1_THREADS) {
            const float v = q < m ? (x[i0 + q] - mhi) - mlo : 0.f;
            S.xa2[q] = make_float2(v, v);
            zs += v;
        }
        const float shift = mu[cbase];
        const int64_t nser = (int64_t)N + m - 1;
        for (int p = t; p < P1_H + mpad + 8; p += P1_THREADS) {
            const int64_t g = (int64_t)cbase + p, g2 = g + P1_H;
            S.xb2[bpad(p)] = make_float2((g < nser ? x[g] : x[nser - 1]) - shift,
                                         (g2 < nser ? x[g2] : x[nser - 1]) - shift);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) zs += __shfl_xor_sync(0xffffffffu, zs, o);
        const float zsum = zs;
        __syncwarp();
        float2 cov[P1_GPT];
        {
            float2 acc[P1_GPT], part[P1_GPT], bb[4];
#pragma unroll
            for (int k = 0; k < P1_GPT; ++k) {
                acc[k] = make_float2(0.f, 0.f);
                bb[k] = S.xb2[bpad(c0 + k)];
            }
            for (int qb = 0; qb < mpad; qb += P1_SUMBLK) {
#pragma unroll
                for (int k = 0; k < P1_GPT; ++k) part[k] = make_float2(0.f, 0.f);
                const int qe = min(mpad, qb + P1_SUMBLK);
                for (int q0 = qb; q0 < qe; q0 += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const float2 a2 = S.xa2[q0 + u];
#pragma unroll
                        for (int k = 0; k < P1_GPT; ++k)
                            part[k] = __ffma2_rn(a2, bb[(u + k) & 3], part[k]);
                        bb[u] = S.xb2[bpad(c0 + q0 + u + 4)];
                    }
                }
#pragma unroll
                for (int k = 0; k < P1_GPT; ++k) acc[k] = __fadd2_rn(acc[k], part[k]);
            }
            // cov = acc - (mu_j - s) * zsum; the start columns' offsets |mu_j - s|
            // (plus the rounding of the FP32 mean) and means for the bound
            float omax = 0.f, umax = 0.f;
#pragma unroll
            for (int k = 0; k < P1_GPT; ++k) {
                const int ja = cbase + c0 + k, jb = ja + P1_H;
                const float mua = ja < N ? mu[ja] : shift;
                const float mub = jb < N ? mu[jb] : shift;
                cov[k] = make_float2(fmaf(-(mua - shift), zsum, acc[k].x),
                                     fmaf(-(mub - shift), zsum, acc[k].y));
                omax = fmaxf(omax, fmaxf(fabsf(mua - shift) + 2.f * kU * fabsf(mua),
                                         fabsf(mub - shift) + 2.f * kU * fabsf(mub)));
                umax = fmaxf(umax, fmaxf(fabsf(mua), fabsf(mub)));
            }
            omax = warp_max(omax);
            umax = warp_max(umax);
            const float n0 = norm_up(wst[i0].w);
            // ---- columns: update terms and inverse norms, maxima
            __syncwarp(); // xa2 / xb2 are overwritten by the column pairs
            float nc = 0.f, fc = 0.f, gc = 0.f;
            for (int q = t; q < R + P1_H; q += P1_THREADS) {
                const float4 a = wst[cbase + q], b = wst[cbase + q + P1_H];
                S.colxy[csw(q)] = make_float4(a.x, b.x, a.y, b.y);
                S.colz[csw(q)] = make_float2(a.z, b.z);
                nc = fmaxf(nc, fmaxf(a.w, b.w));
                fc = fmaxf(fc, fmaxf(fabsf(a.x), fabsf(b.x)));
                gc = fmaxf(gc, fmaxf(fabsf(a.y), fabsf(b.y)));
            }
            nr = norm_up(warp_max(nr));
            fr = warp_max(fr);
            gr = warp_max(gr);
            nc = norm_up(warp_max(nc));
            fc = warp_max(fc);
            gc = warp_max(gc);
            // |x_j - s| = sqrt(n_j^2 + m (mu_j - s)^2) <= n_j + sqrt(m) |mu_j - s|
            const float bmax = (nc + sqrtm * omax) * (1.f + 4.f * kU);
            const float b_start =
                n0 * ((2.f * g_dot + 8.f * kU) * bmax + 2.f * g_z * kU * sqrtm * umax);
            // per-step bound, the comparison's, and the first subtraction
            const float step = kU * (2.f * nr * nc + 4.f * (fc * gr + fr * gc));
            const float dsub = 1.01f * (32.f * step + 2.f * kU * nr * nc);
            const float first = 1.01f * (b_start + 6.f * kU * nr * nc);
#pragma unroll
            for (int k = 0; k < P1_GPT; ++k)
                cov[k] = make_float2(cov[k].x - first, cov[k].y - first);
            __syncwarp();
            // ---- walk the R rows
            if (t == 0) atomicAdd(walked, 1);
            const int lim = N - cbase; // column q is a window iff q < lim
            const bool bound = (rows < R) || (R + P1_D > lim);
            if (bound && thr < 0.f) p1_walk<true>(S, cov, R, rows, lim, dsub, t);
            else p1_walk<false>(S, cov, R, rows, lim, dsub, t);
        }
        __syncwarp();
        // ---- flush pruning marks
        for (int s = t; s < rows; s += P1_THREADS)
            if (S.rowflag[s]) alive[i0 + s] = 0;
        const int lim = N - cbase;
        for (int q = t; q < R + P1_D; q += P1_THREADS)
            if (S.colflag[q] && q < lim) alive[cbase + q] = 0;
        __syncwarp();
    }
}

} // namespace

size_t paddi_phase1_smem(int R, int m)
{
    const int mpad = (m + 7) & ~7;
    const int ncp = p1_ncp(R);
    size_t b = sizeof(float4) * (size_t)R; // rowdg
    const size_t ubytes = std::max((size_t)24 * ncp, (size_t)8 * (mpad + p1_nbp(m)));
    b += (ubytes + 15) & ~(size_t)15;        // colxy + colz / xa2 + xb2
    b += (size_t)(R + P1_D) + (size_t)R;     // flags
    return (b + 15) & ~(size_t)15;
}

cudaError_t paddi_launch_phase1_dev(const float *x, const float4 *wst, const float *mu,
                                    const double *mu64, uint8_t *alive, int32_t N, int32_t m,
                                    int32_t R, int32_t max_chunks, float thr, int32_t row_lo,
                                    int32_t row_hi, int32_t *task_counter, int32_t *walked,
                                    int32_t num_sms, cudaStream_t st)
{
    if (R < 64 || R > 4096 || (R & 7) || m > P1_MAXM || max_chunks < 1 || row_lo < 0 ||
        row_hi > N || row_lo >= row_hi)
        return cudaErrorInvalidValue;
    const size_t smem = paddi_phase1_smem(R, m);
    cudaError_t e = paddi_raise_smem_limit((const void *)k_phase1, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase1, P1_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int nseg = (row_hi - row_lo + R - 1) / R;
    int grid = num_sms * per_sm;
    if (grid > nseg * max_chunks) grid = nseg * max_chunks;
    k_phase1<<<grid, P1_THREADS, smem, st>>>(x, wst, mu, mu64, alive, N, m, R, max_chunks, thr,
                                             row_lo, row_hi, task_counter, walked);
    return cudaGetLastError();
}
