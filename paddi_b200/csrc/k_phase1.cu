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
//   * a task is R rows x 1024 diagonals; each thread owns 8 consecutive
//     diagonals and walks all R rows with the centred covariance update
//         cov(i+1, j+1) = cov(i, j) + df_i dg_j + df_j dg_i
//     (no shared-memory traffic per pair: the 8 column operands rotate
//     through a register ring, one 16-byte load per step);
//   * the starting covariances of the 1024 diagonals are m-term dot products
//     of the centred first row window with the shifted series;
//   * pruned rows are found with one warp ballot per step, pruned columns
//     through shared-memory byte flags; both are flushed as byte stores of 0
//     to the global alive[] array (idempotent, so no atomics).
// Pruning uses rho > thr_prune where thr_prune = 1 - r^2/(2m) + guard, so a
// window is pruned only when its FP32 correlation clears the threshold by
// more than the rounding bound; everything else stays a candidate and is
// settled by the refine and the FP64 recheck.
#include "paddi_internal.cuh"

namespace {

constexpr int P1_THREADS = 128;
constexpr int P1_DPT = 8;                      // diagonals per thread
constexpr int P1_D = P1_THREADS * P1_DPT;      // diagonals per chunk
constexpr int P1_MAXM = 1024;

__device__ __forceinline__ int cpad(int q) { return q + (q >> 3); } // float4 index, conflict-free stride-8
__device__ __forceinline__ int xpad(int p) { return p + (p >> 5); } // float index, conflict-free stride-8

struct P1Smem {
    float4 *roww;  // R
    float4 *colw;  // cpad(R + D)
    float *xa;     // mpad
    float *xb;     // xpad(D + mpad + 8)
    uint8_t *colflag; // R + D
    uint8_t *rowflag; // R
};

template <bool FLATS, bool BOUND>
__device__ __forceinline__ void p1_walk(const P1Smem &S, float (&cov)[P1_DPT], int R, int rows,
                                        int lim, float thr, int t)
{
    const int lane = threadIdx.x & 31;
    float4 ring[P1_DPT];
#pragma unroll
    for (int k = 0; k < P1_DPT; ++k) ring[k] = S.colw[cpad(8 * t + k)];
    uint32_t colbits = 0;
    for (int s0 = 0; s0 < R; s0 += 8) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int s = s0 + u;
            const float4 ri = S.roww[s];
            bool rh = false;
#pragma unroll
            for (int k = 0; k < P1_DPT; ++k) {
                const float4 cj = ring[(u + k) & 7];
                float rho;
                if (FLATS) rho = fmaf(cov[k] * ri.z, cj.z, ri.w * cj.w);
                else rho = cov[k] * ri.z * cj.z;
                bool h = rho > thr;
                if (BOUND) h = h && (s < rows) && (s + 8 * t + k < lim);
                rh |= h;
                colbits |= (uint32_t)h << ((u + k) & 7);
                cov[k] = fmaf(ri.x, cj.y, fmaf(cj.x, ri.y, cov[k]));
            }
            if (__ballot_sync(0xffffffffu, rh) && lane == 0) S.rowflag[s] = 1;
            if ((colbits >> u) & 1u) S.colflag[s + 8 * t] = 1;
            colbits &= ~(1u << u);
            ring[u] = S.colw[cpad(s + 8 * t + 8)];
        }
    }
#pragma unroll
    for (int k = 0; k < P1_DPT; ++k)
        if ((colbits >> k) & 1u) S.colflag[R + 8 * t + k] = 1;
}

__global__ void __launch_bounds__(P1_THREADS)
k_phase1(const float *__restrict__ x, const float4 *__restrict__ wst, const float *__restrict__ mu,
         uint8_t *alive, int32_t N, int32_t m, int32_t R, int32_t max_chunks, float thr,
         const int32_t *__restrict__ flat_count, int32_t *task_counter)
{
    const bool flats = *flat_count > 0;
    extern __shared__ __align__(16) unsigned char p1_smem[];
    const int mpad = (m + 7) & ~7;
    P1Smem S;
    S.roww = reinterpret_cast<float4 *>(p1_smem);
    S.colw = S.roww + R;
    S.xa = reinterpret_cast<float *>(S.colw + cpad(R + P1_D) + 1);
    S.xb = S.xa + mpad;
    S.colflag = reinterpret_cast<uint8_t *>(S.xb + xpad(P1_D + mpad + 8) + 1);
    S.rowflag = S.colflag + R + P1_D;
    __shared__ int s_task;
    __shared__ float s_red[P1_THREADS / 32];

    const int t = threadIdx.x;
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
        // ---- stage rows, columns, and the series slices for the start dots
        for (int s = t; s < R; s += P1_THREADS) {
            S.roww[s] = wst[i0 + s]; // zero beyond N (padded tail)
            S.rowflag[s] = 0;
        }
        const int cbase = i0 + d0;
        for (int q = t; q < R + P1_D; q += P1_THREADS) {
            S.colw[cpad(q)] = wst[cbase + q];
            S.colflag[q] = 0;
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

        // ---- starting covariances of diagonals d0 + 8t + k at row i0
        float cov[P1_DPT];
#pragma unroll
        for (int k = 0; k < P1_DPT; ++k) cov[k] = 0.f;
        {
            float b[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) b[k] = S.xb[xpad(8 * t + k)];
            for (int q0 = 0; q0 < mpad; q0 += 8) {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const float a = S.xa[q0 + u];
#pragma unroll
                    for (int k = 0; k < P1_DPT; ++k) cov[k] = fmaf(a, b[(u + k) & 7], cov[k]);
                    b[u] = S.xb[xpad(8 * t + q0 + u + 8)];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < P1_DPT; ++k) {
            const int j = cbase + 8 * t + k;
            const float muj = j < N ? mu[j] : shift;
            cov[k] = fmaf(-(muj - shift), zsum, cov[k]);
        }
        // ---- walk the R rows
        const int lim = N - cbase; // column q is a window iff q < lim
        const bool bound = (rows < R) || (R + P1_D > lim);
        if (flats) {
            if (bound && thr < 0.f) p1_walk<true, true>(S, cov, R, rows, lim, thr, t);
            else p1_walk<true, false>(S, cov, R, rows, lim, thr, t);
        } else {
            if (bound && thr < 0.f) p1_walk<false, true>(S, cov, R, rows, lim, thr, t);
            else p1_walk<false, false>(S, cov, R, rows, lim, thr, t);
        }
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
    auto cpadh = [](int q) { return q + (q >> 3); };
    auto xpadh = [](int p) { return p + (p >> 5); };
    size_t b = 0;
    b += sizeof(float4) * (size_t)R;
    b += sizeof(float4) * (size_t)(cpadh(R + P1_D) + 1);
    b += sizeof(float) * (size_t)mpad;
    b += sizeof(float) * (size_t)(xpadh(P1_D + mpad + 8) + 1);
    b += (size_t)(R + P1_D) + (size_t)R;
    return (b + 15) & ~(size_t)15;
}

cudaError_t paddi_launch_phase1_dev(const float *x, const float4 *wst, const float *mu,
                                    uint8_t *alive, int32_t N, int32_t m, int32_t R,
                                    int32_t max_chunks, float thr_prune,
                                    const int32_t *flat_count, int32_t *task_counter,
                                    int32_t num_sms, cudaStream_t st)
{
    if (R < 64 || R > 2048 || (R & 7) || m > P1_MAXM || max_chunks < 1)
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
                                             flat_count, task_counter);
    return cudaGetLastError();
}
