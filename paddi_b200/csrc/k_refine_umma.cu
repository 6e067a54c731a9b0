// k_refine_umma.cu -- dense candidate refine on tcgen05 tensor cores with
// three-term split 16-bit operands (hi*hi + hi*lo + lo*hi, FP32 accumulate).
//
// Reference: gpu_global_discords_refine (src/PD3_kernels.cuh:582-662), a
// 32x32-tiled FP32 SGEMM of a host-gathered candidate matrix against the
// Hankel windows of the series.  Same contraction here, mapped onto UMMA:
//
//   D[(c,b), a] = sum_k' A[(c,b), k'] * B[a, k']       M = 128, N = 256, K' = m+7 rounded to 16
//   A[(c,b), k'] = zhat_c[k' - b]    (16 candidates x 8 shifted copies, zero padded)
//   B[a, k']     = y[8a + k']        (y = scaled series slice minus a shift)
// so D[(c,b), a] = <zhat_c, y[j .. j+m)> for window j = j0 + 8a + b: one tile
// covers 16 candidates x 2048 windows.
//
// The Hankel operand is never expanded: with SWIZZLE_NONE a K-major core
// matrix is 8 rows of 16 bytes, and the rows of B are 8 elements (16 bytes)
// apart in the series, so the descriptor of B is the raw series slice with
// leading-byte offset 16 and stride-byte offset 128.  The 8 shifts live on
// the candidate side instead, where the operand stays resident for a whole
// work item.
//
// Precision: zhat is normalised (|zhat| = 1) and scaled by 2^8, the slice is
// shifted by x[j0] and scaled by a power of two that puts its largest
// magnitude just below 2^14; both are split into hi + lo 16-bit halves.  The
// rounding of the slice is amplified by |x - shift| / sigma_window, which is
// why FP16 (11-bit mantissa, ~2^-22 per split value) is the default element
// type; BF16 (8-bit mantissa, ~2^-17) is available as the alternative.  The
// epilogue removes the shift exactly with the candidate's sum of split
// values: rho = (D 2^-(8+e) - sum(zhat') (mu_j - shift)) inv_j.
//
// Layout of the work.  Tiles sit on a fixed grid of 2048-window blocks.  Once
// per length, k_tile_prep converts every block's slice into its hi / lo
// halves and its per-window epilogue data (inv_j 2^-(8+e), (mu_j - shift)
// inv_j) in global memory (L2-resident).  The refine is then a pipeline of
// roles inside one persistent CTA per SM, coupled only by mbarriers:
//   * loader (one thread): bulk async copies (cp.async.bulk, no multicast)
//     of the next tile's slice into one of two shared-memory stages, and of
//     the current tile's window data;
//   * MMA issuer (one thread): 3 x K'/16 tcgen05.mma of 128x256x16 per tile
//     into one of two TMEM accumulators (all 512 columns), then commit;
//   * epilogue (8 warps, two per TMEM lane quarter, 128 columns each):
//     double-buffered tcgen05.ld, rho with packed f32x2 FMAs, running maxima,
//     prune flags.
// The candidate operand is built by all 384 threads at the start of a work
// item.  When every candidate of the item is pruned the loader stops and
// sends an end token through the pipeline, so all roles consume the same
// barrier phases.  Every mbarrier wait is bounded; on timeout the kernel
// records status 3, waits (bounded) for its own copies and MMAs, releases
// its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <float.h>

#include <cmath>

#include "paddi_internal.cuh"

using paddi::f2ord;

namespace {

constexpr int UM_THREADS = 384;  // 12 warps
constexpr int UM_TCMAX = 16;     // candidates per tile (M = 128); 8 for M = 64
constexpr int UM_N = 256;        // windows at stride 8
constexpr int UM_TW = UM_N * 8;  // windows per tile (one block of the grid)
constexpr int UM_WAVES = 1;      // work items per CTA and round when candidate tiles are few
constexpr int UM_KMAX128 = 368;  // largest K' with M = 128 (shared-memory bound)
constexpr int UM_KMAX64 = 736;   // largest K' with M = 64
constexpr int ZSCALE = 8;        // zhat scaled by 2^8 before splitting
constexpr int WD_ROW = 129;      // float4 entries per shift row of the window data (128 + pad)
constexpr int WD_BYTES = 8 * WD_ROW * 16;
// limit of the abort path's drain waits (~2 s at 1.9 GHz): copies and MMAs the
// kernel issued complete on their own, so these waits end long before it
constexpr long long kDrainCycles = 4000000000ll;
constexpr int EPI_WARP0 = 4;     // warps 4..11: epilogue (two per TMEM lane quarter)
constexpr int EPI_WARPS = 8;
constexpr int MMA_WARP = 0, LOAD_WARP = 1;

__host__ __device__ constexpr int kpad_of(int m) { return ((m + 7) + 15) & ~15; }
__host__ __device__ constexpr int slice_cnt(int kp) { return UM_TW + kp + 16; }
// scratch row stride (32-bit words) of the candidate operand build: 4 words of
// front padding + kp/2 words, rounded up to 8 modulo 32
__host__ __device__ constexpr int zrow_words(int kp)
{
    return (4 + kp / 2) + ((8 - (4 + kp / 2) % 32) + 32) % 32;
}

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of the phase with the given parity;
// false when `limit` clock cycles passed first.
__device__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bulk async copy global -> this CTA's shared memory (no multicast), completing
// `bytes` transaction bytes on bar.  dst, src 16-byte aligned; bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
                 "%2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, SWIZZLE_NONE, K-major, sm100 version bits.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::f16, D = F32, A/B = fmt (0 F16, 1 BF16), K-major, M, N.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t fmt, int M, int N)
{
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u),
        "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

// tcgen05.ld without the wait, and a wait that is tied to the destination
// registers (so no use of them can be scheduled before it).
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                 "[%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                   "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                   "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[32])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                   "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                   "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                   "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}

// max(a, b, c) in one instruction (sm_100 three-input form)
__device__ __forceinline__ float fmax3(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// ------------------------------------------------------------------ element types
template <bool BF> struct E16;
template <> struct E16<false> {
    using T = __half;
    static constexpr uint32_t fmt = 0;
    __device__ static __half cvt(float v) { return __float2half_rn(v); }
    __device__ static float back(__half v) { return __half2float(v); }
};
template <> struct E16<true> {
    using T = __nv_bfloat16;
    static constexpr uint32_t fmt = 1;
    __device__ static __nv_bfloat16 cvt(float v) { return __float2bfloat16_rn(v); }
    __device__ static float back(__nv_bfloat16 v) { return __bfloat162float(v); }
};

// ------------------------------------------------------------------ tile prep
// Block b (windows [2048 b, 2048 b + 2048)): slice x[j0 .. j0 + cnt) minus
// its level s, scaled by 2^e (largest magnitude just below 2^14), split
// into hi and lo halves: bq[b * 2cnt ...] = hi, then lo.  Window data for the
// epilogue in its read layout: shift row s = q % 8, column pair k = q / 16,
// slot = (q / 8) % 2: wd[s * 129 + k] = {a(slot 0), a(slot 1), b(slot 0), b(slot 1)}
// with a = inv_j 2^-(8+e) and b = (mu_j - s) inv_j (zero past N).
// Rounding bound: window j's correlations carry at most g_j = window_bound()
// (E A_j + F inv_j); g_j grows with |mu_j - s| / |x_j - mu_j|.  The level s
// is the mean of the block's window means weighted by 1 / |x_j - mu_j|^2 (it
// minimises the sum of (mu_j - s)^2 / |x_j - mu_j|^2, so the low-variance
// windows, where the amplification is large, pull it towards their level);
// the slice's midrange if no window has a norm.  A window with g_j > gcap is
// "fragile": its a is NaN
// (the epilogue's maxima skip it) and it is appended to frag_list, whose
// pairs are evaluated in FP64 later.  The largest g_j of the block's other
// windows, G, is stored in the padding entry wd[128].x: the epilogue
// subtracts it from every correlation of the tile (a lower bound that is safe
// to prune on) and adds it back to the maxima it keeps (the middle of the
// interval, within gcap of every true value).
constexpr int TP_THREADS = 256;

template <bool BF>
__global__ void __launch_bounds__(TP_THREADS)
k_tile_prep(const float *__restrict__ x, int64_t nser, int32_t cnt, int32_t m,
            const float4 *__restrict__ wst, const float *__restrict__ mu, uint16_t *__restrict__ bq,
            float4 *__restrict__ wdq, float E, float Fu, float gcap, int32_t *frag_list,
            int32_t *frag_count)
{
    using X = E16<BF>;
    __shared__ float red[4][TP_THREADS / 32];
    const int b = blockIdx.x;
    const int64_t j0 = (int64_t)b * UM_TW;
    const int64_t N = nser - m + 1;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float sw = 0.f, swm = 0.f; // sums of 1/|x_j - mu_j|^2 and mu_j/|x_j - mu_j|^2
    for (int q = threadIdx.x; q < UM_TW; q += TP_THREADS) {
        const int64_t j = j0 + q;
        if (j < N) {
            const float iv = wst[j].z;
            const float wgt = fminf(iv * iv, 1e30f);
            sw += wgt;
            swm = fmaf(wgt, mu[j], swm);
        }
    }
    float lo_v = INFINITY, hi_v = -INFINITY;
    for (int p = threadIdx.x; p < cnt; p += TP_THREADS) {
        const int64_t g = j0 + p;
        if (g < nser) {
            lo_v = fminf(lo_v, x[g]);
            hi_v = fmaxf(hi_v, x[g]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo_v = fminf(lo_v, __shfl_xor_sync(0xffffffffu, lo_v, o));
        hi_v = fmaxf(hi_v, __shfl_xor_sync(0xffffffffu, hi_v, o));
        sw += __shfl_xor_sync(0xffffffffu, sw, o);
        swm += __shfl_xor_sync(0xffffffffu, swm, o);
    }
    if (lane == 0) {
        red[0][w] = lo_v;
        red[1][w] = hi_v;
        red[2][w] = sw;
        red[3][w] = swm;
    }
    __syncthreads();
    lo_v = INFINITY;
    hi_v = -INFINITY;
    sw = 0.f;
    swm = 0.f;
#pragma unroll
    for (int k = 0; k < TP_THREADS / 32; ++k) {
        lo_v = fminf(lo_v, red[0][k]);
        hi_v = fmaxf(hi_v, red[1][k]);
        sw += red[2][k];
        swm += red[3][k];
    }
    __syncthreads();
    float sh = 0.5f * lo_v + 0.5f * hi_v; // midrange (j0 < nser always)
    if (sw > 0.f) {
        const float lv = swm / sw; // the weighted level, kept inside the slice's range
        if (isfinite(lv)) sh = fminf(fmaxf(lv, lo_v), hi_v);
    }
    const float mx = fmaxf(fabsf(hi_v - sh), fabsf(lo_v - sh));
    int e = 0;
    if (mx > 0.f) {
        int ex;
        frexpf(mx, &ex); // mx = f * 2^ex, f in [0.5, 1)
        e = 14 - ex;     // mx * 2^e < 2^14
        e = max(-100, min(100, e));
    }
    const float sc = ldexpf(1.f, e);
    const float dsc = ldexpf(1.f, -(ZSCALE + e));
    uint32_t *hi = reinterpret_cast<uint32_t *>(bq + (size_t)b * 2 * cnt);
    uint32_t *lo = reinterpret_cast<uint32_t *>(bq + (size_t)b * 2 * cnt + cnt);
    for (int p2 = threadIdx.x; p2 < cnt / 2; p2 += TP_THREADS) {
        const int64_t g = j0 + 2 * p2;
        const float u0 = (g < nser ? x[g] - sh : 0.f) * sc;
        const float u1 = (g + 1 < nser ? x[g + 1] - sh : 0.f) * sc;
        const typename X::T h0 = X::cvt(u0), h1 = X::cvt(u1);
        const typename X::T l0 = X::cvt(u0 - X::back(h0)), l1 = X::cvt(u1 - X::back(h1));
        hi[p2] = (uint32_t)reinterpret_cast<const uint16_t &>(h0) |
                 ((uint32_t)reinterpret_cast<const uint16_t &>(h1) << 16);
        lo[p2] = (uint32_t)reinterpret_cast<const uint16_t &>(l0) |
                 ((uint32_t)reinterpret_cast<const uint16_t &>(l1) << 16);
    }
    float *wf = reinterpret_cast<float *>(wdq + (size_t)b * 8 * WD_ROW);
    const float F = Fu * mx, fm = (float)m;
    float gmax = 0.f;
    for (int q = threadIdx.x; q < UM_TW; q += TP_THREADS) {
        const int64_t j = j0 + q; // the padded tail beyond N is zero
        const float iv = wst[j].z, mv = mu[j];
        const float g = paddi::window_bound(iv, mv, sh, fm, E, F);
        const bool frag = j < N && g > gcap;
        if (!frag) gmax = fmaxf(gmax, g);
        const int s = q & 7, i = q >> 3, k = i >> 1, slot = i & 1;
        wf[(s * WD_ROW + k) * 4 + slot] = frag ? __int_as_float(0x7fffffff) : iv * dsc;
        wf[(s * WD_ROW + k) * 4 + 2 + slot] = (mv - sh) * iv;
        // fragile windows in index order within each warp (runs stay contiguous)
        const unsigned bal = __ballot_sync(0xffffffffu, frag);
        if (bal) {
            int base = 0;
            if (lane == 0) base = atomicAdd(frag_count, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (frag) frag_list[base + __popc(bal & ((1u << lane) - 1u))] = (int32_t)j;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gmax = fmaxf(gmax, __shfl_xor_sync(0xffffffffu, gmax, o));
    if (lane == 0) red[0][w] = gmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        float G = 0.f;
        for (int k = 0; k < TP_THREADS / 32; ++k) G = fmaxf(G, red[0][k]);
        wf[(0 * WD_ROW + 128) * 4] = G; // padding entry of shift row 0
    }
}

// ------------------------------------------------------------------ shared memory
struct UmLayout {
    uint32_t a_hi, a_lo, b[2][2], wd, bytes;
};

__host__ __device__ inline UmLayout um_layout(int MM, int kp)
{
    UmLayout L;
    const uint32_t a_bytes = (uint32_t)MM * kp * 2;
    const uint32_t b_bytes = (uint32_t)slice_cnt(kp) * 2; // multiple of 32
    L.a_hi = 0;
    L.a_lo = a_bytes;
    uint32_t o = 2 * a_bytes;
    for (int s = 0; s < 2; ++s)
        for (int h = 0; h < 2; ++h) {
            L.b[s][h] = o;
            o += b_bytes;
        }
    L.wd = o; // window data of the current tile, directly after the stages
    o += WD_BYTES;
    L.bytes = o;
    return L;
}

struct UmShared {
    uint64_t full_b[2];    // loader -> MMA: stage holds the tile's slice (or an end token)
    uint64_t mma_done[2];  // tcgen05.commit: the tile's MMAs are complete
    uint64_t acc_empty[2]; // epilogue -> MMA: accumulator drained
    uint64_t wd_full;      // loader -> epilogue: window data of the tile (or an end token)
    uint64_t wd_empty;     // epilogue -> loader: window data consumed
    uint64_t drain;        // final MMA drain on abort
    // absolute phase index of the last arrival the loader issued on full_b[s] /
    // wd_full (-1: none yet); the abort path waits only for those
    int last_full[2], last_wd;
    uint32_t tmem_base;
    int item, abort, tok;
    int built_tile; // candidate tile whose operand sits in A (-1: none)
    volatile int item_dead;
    int tile_live; // live candidates at the start of the current tile (instrumentation)
    volatile int vb[2], vw;
    int cw[UM_TCMAX], cp[UM_TCMAX];
    float cflat[UM_TCMAX], zsum[UM_TCMAX];
    uint32_t rmax[UM_TCMAX];
    volatile uint8_t dead[UM_TCMAX];
};

// Completed phases of each barrier before the current work item.
struct UmPhases {
    uint32_t full[2], done[2], acc[2], wdf, wde;
};

__device__ __forceinline__ uint32_t par(uint32_t idx) { return idx & 1u; }

// MM = 128: 16 candidates, accumulator row r in TMEM lane r.
// MM = 64:  8 candidates, accumulator row r in TMEM lane (r % 16) + 32 (r / 16)
//           (lanes 16..31 of every subpartition stay unused).
template <bool BF, int MM>
__global__ void __launch_bounds__(UM_THREADS, 1)
k_refine_umma(const float *__restrict__ x, const float4 *__restrict__ wst,
              const float *__restrict__ mu, const int32_t *__restrict__ cand,
              const int32_t *__restrict__ list, const int32_t *__restrict__ list_count,
              const uint16_t *__restrict__ bq, const float4 *__restrict__ wdq,
              PaddiAttemptDev *att, int32_t *work, uint32_t *rho_max, uint8_t *pruned, int32_t N,
              int32_t m, int32_t jb, int32_t je, float thr, int32_t grid_ctas, long long wl,
              int32_t withhold, int32_t round, int32_t je_all)
{
    using X = E16<BF>;
    constexpr int UM_M = MM;
    constexpr int UM_TC = MM / 8;
    constexpr int RG = MM / 8;          // 8-row core-matrix groups of A
    extern __shared__ __align__(1024) unsigned char um_smem[];
    __shared__ UmShared S;
    const int kp = kpad_of(m);
    const int cnt = slice_cnt(kp);
    const UmLayout L = um_layout(MM, kp);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    const int C = *list_count;
    // an earlier round with one candidate tile left took every remaining window
    const int cov = att->covered_from;
    if (C <= 0 || je <= jb || (cov > 0 && cov <= round)) return; // uniform, before any TMEM use
    // one tile left: later rounds could not shrink it, so take the rest of the
    // windows now and spare them their launches' fixed cost
    if (C <= UM_TC && je_all > je) {
        je = je_all;
        if (blockIdx.x == 0 && threadIdx.x == 0) att->covered_from = round + 1;
    }

    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&S.full_b[s], 1);
            mbar_init(&S.mma_done[s], 1);
            mbar_init(&S.acc_empty[s], EPI_WARPS);
        }
        mbar_init(&S.wd_full, 1);
        mbar_init(&S.wd_empty, EPI_WARPS);
        mbar_init(&S.drain, 1);
        S.abort = 0;
        S.built_tile = -1;
        S.last_full[0] = S.last_full[1] = S.last_wd = -1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&S.tmem_base)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;
    UmPhases ph = {{0u, 0u}, {0u, 0u}, {0u, 0u}, 0u, 0u};
    bool mma_issued = false; // MMA thread: any MMA issued

    const int range = je - jb;
    const int tiles = (C + UM_TC - 1) / UM_TC;
    // at most UM_WAVES items per CTA when the candidate tiles are few, items of
    // at least one 2048-window block
    const int splits = max(1, min(range / UM_TW, (UM_WAVES * grid_ctas) / tiles));
    const int span = (((range + splits - 1) / splits) + UM_TW - 1) / UM_TW * UM_TW;
    const int total = tiles * splits;
    const uint32_t idesc = idesc_f16(X::fmt, UM_M, UM_N);
    const uint32_t a_hi_s = smem_u32(um_smem + L.a_hi), a_lo_s = smem_u32(um_smem + L.a_lo);
    const int kblocks = kp / 16;
    // epilogue geometry: lane group g (TMEM lanes 32g..32g+31)
    const int g = warp & 3, hcol = (warp - EPI_WARP0) >> 2; // lane quarter, column half
    const bool rowok = MM == 128 || lane < 16;
    const int row = MM == 128 ? 32 * g + lane : 16 * g + (lane & 15);
    const int cidx = row >> 3, bsh = row & 7;
    const float4 *wd4 = reinterpret_cast<const float4 *>(um_smem + L.wd);

    for (;;) {
        if (threadIdx.x == 0) S.item = atomicAdd(work, 1);
        __syncthreads();
        const int item = S.item;
        if (item >= total || S.abort) break;
        const int tile = item % tiles, split = item / tiles;
        const int j_lo = jb + split * span, j_hi = min(je, j_lo + span);
        if (threadIdx.x < UM_TC) {
            const int li = tile * UM_TC + threadIdx.x;
            const bool v = li < C;
            const int pos = v ? list[li] : 0;
            const int w = v ? cand[pos] : 0;
            S.cw[threadIdx.x] = w;
            S.cp[threadIdx.x] = pos;
            S.dead[threadIdx.x] = !v || __ldcg(pruned + pos);
            S.cflat[threadIdx.x] = (v && wst[w].z == 0.f) ? 1.f : 0.f; // flat candidate
            S.rmax[threadIdx.x] = f2ord(-INFINITY);
        }
        if (threadIdx.x == 0) {
            S.item_dead = 0;
            S.tok = -1;
        }
        __syncthreads();
        {
            int a = threadIdx.x < UM_TC ? !S.dead[threadIdx.x] : 0;
            if (!__syncthreads_or(a) || j_lo >= j_hi) continue; // all threads agree
        }
        if (threadIdx.x == 32) { // read by the epilogue after the barriers below
            int alive = 0;
            for (int c = 0; c < UM_TC; ++c) alive += !S.dead[c];
            S.tile_live = alive;
        }
        const int T = (j_hi - j_lo + UM_TW - 1) / UM_TW;
        const int blk0 = j_lo / UM_TW; // j_lo is a multiple of UM_TW
        // the first tile's slice streams into stage 0 while the operand is built
        // (the build's scratch is stage 1 + the window data)
        if (warp == LOAD_WARP && lane == 0) {
            S.vb[0] = 1;
            // test hook (withhold != 0): the CTA holding work item 0 never fills
            // its first stage, so the MMA thread's wait runs out; nothing is in flight
            const bool skip = withhold && item == 0;
            if (!skip) {
                const uint16_t *src = bq + (size_t)blk0 * 2 * cnt;
                mbar_arrive_expect_tx(&S.full_b[0], (uint32_t)(4 * cnt));
                bulk_g2s(um_smem + L.b[0][0], src, (uint32_t)(2 * cnt), &S.full_b[0]);
                bulk_g2s(um_smem + L.b[0][1], src + cnt, (uint32_t)(2 * cnt), &S.full_b[0]);
                S.last_full[0] = (int)ph.full[0];
            }
        }
        // ---- candidate operand: 16 x (hi, lo) rows of scaled zhat, then 8 shifted
        //      copies; kept from the CTA's previous item when that had the same
        //      candidate tile (a candidate pruned since then only costs its rows'
        //      work: its results no longer matter)
        if (S.built_tile != tile) {
            // scratch rows of 32-bit words: 4 zero words (8 elements) of front
            // padding, then zhat[0..kp); stride ksw words with ksw % 32 == 8, so
            // the four candidates a warp reads sit in disjoint bank ranges
            const int ksw = zrow_words(kp);
            uint32_t *zhw = reinterpret_cast<uint32_t *>(um_smem + L.b[1][0]);
            uint32_t *zlw = zhw + UM_TC * ksw;
            typename X::T *zh = reinterpret_cast<typename X::T *>(zhw);
            typename X::T *zl = reinterpret_cast<typename X::T *>(zlw);
            const int c = threadIdx.x >> 4, t16 = threadIdx.x & 15;
            const int w = c < UM_TC ? S.cw[c] : 0;
            const bool live = c < UM_TC && !S.dead[c];
            const float muc = live ? mu[w] : 0.f;
            const float ivc = live ? wst[w].z * 256.f : 0.f; // 2^ZSCALE
            float zs = 0.f;
            if (c < UM_TC)
                for (int q = 4 + (kp >> 1) + t16; q < ksw; q += 16) { // tail words
                    zhw[c * ksw + q] = 0u;
                    zlw[c * ksw + q] = 0u;
                }
            if (c < UM_TC && t16 < 4) { // front padding
                zhw[c * ksw + t16] = 0u;
                zlw[c * ksw + t16] = 0u;
            }
            for (int k = t16; k < kp; k += 16) {
                const float v = (live && k < m) ? (x[w + k] - muc) * ivc : 0.f;
                const typename X::T h = X::cvt(v);
                const typename X::T l = X::cvt(v - X::back(h));
                if (c < UM_TC) {
                    zh[c * 2 * ksw + 8 + k] = h;
                    zl[c * 2 * ksw + 8 + k] = l;
                }
                zs += X::back(h) + X::back(l);
            }
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) zs += __shfl_xor_sync(0xffffffffu, zs, o);
            if (t16 == 0 && c < UM_TC) S.zsum[c] = zs * (1.f / 256.f);
            __syncthreads();
            // A[(c,b), k'] = z_c[k' - b] in K-major core matrices:
            // byte offset ((k'/8)*RG + r/8)*128 + (r%8)*16 + (k'%8)*2.
            // Elements k'-b .. k'-b+7 start at padded element p0 = 8 + 8 kc - b:
            // five 32-bit words from word p0/2, funnel-shifted by 16 bits when p0 is odd.
            const int chunks = kp / 8;
            for (int e = threadIdx.x; e < UM_M * chunks; e += UM_THREADS) {
                const int r = e & (UM_M - 1), kc = e / UM_M;
                const int cc = r >> 3, b = r & 7;
                const int p0 = 8 + 8 * kc - b;
                const uint32_t shf = (uint32_t)(p0 & 1) * 16u;
                const uint32_t *rh = zhw + cc * ksw + (p0 >> 1);
                const uint32_t *rl = zlw + cc * ksw + (p0 >> 1);
                uint32_t wh[5], wl[5], ph2[4], pl2[4];
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    wh[q] = rh[q];
                    wl[q] = rl[q];
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ph2[q] = __funnelshift_r(wh[q], wh[q + 1], shf);
                    pl2[q] = __funnelshift_r(wl[q], wl[q + 1], shf);
                }
                const uint32_t off = (uint32_t)((kc * RG + (r >> 3)) * 128 + (r & 7) * 16);
                *reinterpret_cast<uint4 *>(um_smem + L.a_hi + off) =
                    make_uint4(ph2[0], ph2[1], ph2[2], ph2[3]);
                *reinterpret_cast<uint4 *>(um_smem + L.a_lo + off) =
                    make_uint4(pl2[0], pl2[1], pl2[2], pl2[3]);
            }
            fence_proxy_async_smem(); // A for the tensor core; scratch for the bulk copies
            __syncthreads();
            if (threadIdx.x == 0) S.built_tile = tile; // read after the next item's barrier
        }

        // ================================================================ roles
        if (warp == LOAD_WARP && lane == 0) {
            // slice of tile u into stage u&1 (after the MMAs of tile u-2 are done);
            // an end token instead once the item is dead
            auto load_slice = [&](int u) -> bool {
                const int s = u & 1;
                if (u >= 2 && !mbar_wait_bounded(&S.mma_done[s], par(ph.done[s] + ((u - 2) >> 1)), wl))
                    return false;
                S.last_full[s] = (int)(ph.full[s] + (u >> 1));
                if (S.item_dead) {
                    S.vb[s] = 0;
                    S.tok = u;
                    mbar_arrive(&S.full_b[s]);
                    return true;
                }
                S.vb[s] = 1;
                const uint16_t *src = bq + (size_t)(blk0 + u) * 2 * cnt;
                mbar_arrive_expect_tx(&S.full_b[s], (uint32_t)(4 * cnt));
                bulk_g2s(um_smem + L.b[s][0], src, (uint32_t)(2 * cnt), &S.full_b[s]);
                bulk_g2s(um_smem + L.b[s][1], src + cnt, (uint32_t)(2 * cnt), &S.full_b[s]);
                return true;
            };
            bool ok = true; // slice 0 was issued before the operand build
            for (int u = 0; ok && u < T; ++u) {
                if (u + 1 < T) ok = load_slice(u + 1);
                if (!ok) break;
                // window data of tile u (after the epilogue is done with tile u-1)
                if (u >= 1 && !mbar_wait_bounded(&S.wd_empty, par(ph.wde + (u - 1)), wl)) {
                    ok = false;
                    break;
                }
                S.last_wd = (int)(ph.wdf + u);
                if (S.tok == u + 1) { // end token: no window data for tile u either
                    S.vw = 0;
                    mbar_arrive(&S.wd_full);
                    break;
                }
                S.vw = 1;
                mbar_arrive_expect_tx(&S.wd_full, (uint32_t)WD_BYTES);
                bulk_g2s(um_smem + L.wd, wdq + (size_t)(blk0 + u) * 8 * WD_ROW, (uint32_t)WD_BYTES,
                         &S.wd_full);
            }
            if (!ok) S.abort = 1;
        } else if (warp == MMA_WARP && lane == 0) {
            for (int u = 0; u < T; ++u) {
                const int s = u & 1;
                if (!mbar_wait_bounded(&S.full_b[s], par(ph.full[s] + (u >> 1)), wl)) {
                    S.abort = 1;
                    break;
                }
                // the accumulator's previous tile must be drained first, also before an
                // end token: its commit completes a phase of mma_done[s] that the
                // epilogue may still be waiting on for tile u-2
                if (u >= 2 &&
                    !mbar_wait_bounded(&S.acc_empty[s], par(ph.acc[s] + ((u - 2) >> 1)), wl)) {
                    S.abort = 1;
                    break;
                }
                if (!S.vb[s]) { // end token: pass it on (the commit also covers earlier MMAs)
                    umma_commit(&S.mma_done[s]);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(s * UM_N);
                const uint32_t bh = smem_u32(um_smem + L.b[s][0]), bl = smem_u32(um_smem + L.b[s][1]);
                for (int kb = 0; kb < kblocks; ++kb) {
                    // K-block kb = core-matrix columns 2kb, 2kb+1; LBO = next K column of cores
                    const uint64_t ah = sdesc(a_hi_s + kb * (2 * RG * 128), RG * 128, 128);
                    const uint64_t al = sdesc(a_lo_s + kb * (2 * RG * 128), RG * 128, 128);
                    const uint64_t bhd = sdesc(bh + kb * 32, 16, 128);
                    const uint64_t bld = sdesc(bl + kb * 32, 16, 128);
                    umma_f16(d, ah, bhd, idesc, kb > 0 ? 1u : 0u);
                    umma_f16(d, ah, bld, idesc, 1u);
                    umma_f16(d, al, bhd, idesc, 1u);
                }
                umma_commit(&S.mma_done[s]);
                mma_issued = true;
            }
        } else if (warp >= EPI_WARP0) {
            float rmax = -INFINITY;
            const int wc = S.cw[cidx];
            const float zsc = S.zsum[cidx], fc = S.cflat[cidx];
            const float2 nz2 = make_float2(-zsc, -zsc);
            // Every lane waits (acquire) and the warp then agrees through a vote, so
            // the warp is converged and takes the same branch at every tcgen05.ld.
            for (int u = 0; u < T; ++u) {
                const int s = u & 1;
                if (!__all_sync(0xffffffffu, mbar_wait_bounded(&S.wd_full, par(ph.wdf + u), wl))) {
                    S.abort = 1;
                    break;
                }
                const int vw = __shfl_sync(0xffffffffu, S.vw, 0);
                if (!__all_sync(0xffffffffu,
                                mbar_wait_bounded(&S.mma_done[s], par(ph.done[s] + (u >> 1)), wl))) {
                    S.abort = 1;
                    break;
                }
                if (!vw) { // end token; its slice twin at tile u+1 is committed too
                    const int s1 = (u + 1) & 1;
                    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&S.mma_done[s1], par(ph.done[s1] + ((u + 1) >> 1)), wl)))
                        S.abort = 1;
                    break;
                }
                tc_fence_after();
                const int j0 = j_lo + u * UM_TW;
                if (!__shfl_sync(0xffffffffu, S.item_dead, 0)) {
                    const uint32_t tb = tmem + ((uint32_t)(32 * g) << 16) +
                                        (uint32_t)(s * UM_N + 128 * hcol);
                    const bool masked = (j0 + UM_TW > j_hi) ||
                                        (wc > j0 - m + 1 && wc < j0 + UM_TW + m - 1) || fc != 0.f;
                    const float4 *wrow = wd4 + bsh * WD_ROW + 64 * hcol;
                    // the tile's rounding bound (tile prep): correlations are lowered
                    // by it for the prune test and raised back for the kept maxima
                    const float Gt = wd4[128].x;
                    const float2 ng2 = make_float2(-Gt, -Gt);
                    float tm[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
                    // 4 chunks of 32 columns; the load of chunk cb+1 overlaps the math of cb
                    auto chunk = [&](const uint32_t (&r)[32], int cb) {
                        if (!masked) {
#pragma unroll
                            for (int i2 = 0; i2 < 16; ++i2) {
                                const float4 wv = wrow[16 * cb + i2];
                                const float2 dd = make_float2(__uint_as_float(r[2 * i2]),
                                                              __uint_as_float(r[2 * i2 + 1]));
                                const float2 rho = __ffma2_rn(
                                    dd, make_float2(wv.x, wv.y),
                                    __ffma2_rn(nz2, make_float2(wv.z, wv.w), ng2));
                                tm[i2 & 3] = fmax3(tm[i2 & 3], rho.x, rho.y);
                            }
                        } else {
#pragma unroll
                            for (int i = 0; i < 32; ++i) {
                                const int col = 128 * hcol + 32 * cb + i;
                                const int j = j0 + 8 * col + bsh;
                                const float4 wv = wrow[(32 * cb + i) >> 1];
                                const float wa = (i & 1) ? wv.y : wv.x;
                                const float wb = (i & 1) ? wv.w : wv.z;
                                float rho = fmaf(__uint_as_float(r[i]), wa, fmaf(-zsc, wb, -Gt));
                                if (fc != 0.f && wa == 0.f) rho += 1.f; // two flat windows
                                const int dd = wc > j ? wc - j : j - wc;
                                if (j < j_hi && dd >= m - 1) tm[i & 3] = fmaxf(tm[i & 3], rho);
                            }
                        }
                    };
                    uint32_t ra[32], rb[32];
                    tmem_ld32_async(tb, ra);
                    tmem_wait_ld(ra);
                    tmem_ld32_async(tb + 32, rb);
                    chunk(ra, 0);
                    tmem_wait_ld(rb);
                    tmem_ld32_async(tb + 64, ra);
                    chunk(rb, 1);
                    tmem_wait_ld(ra);
                    tmem_ld32_async(tb + 96, rb);
                    chunk(ra, 2);
                    tmem_wait_ld(rb);
                    chunk(rb, 3);
                    float tmax = fmaxf(fmaxf(tm[0], tm[1]), fmaxf(tm[2], tm[3]));
                    if (!rowok) tmax = -INFINITY;
                    rmax = fmaxf(rmax, tmax + Gt); // the interval's middle (-inf stays)
                    const unsigned bal = __ballot_sync(0xffffffffu, tmax > thr);
                    if (lane < UM_TC / 4) {
                        const int ci = (UM_TC / 4) * g + lane;
                        if (!S.dead[ci]) {
                            if ((bal >> (8 * lane)) & 0xFFu) {
                                S.dead[ci] = 1;
                                pruned[S.cp[ci]] = 1;
                            } else if (__ldcg(pruned + S.cp[ci])) {
                                S.dead[ci] = 1; // pruned by another CTA's item
                            }
                        }
                    }
                    __syncwarp();
                    if (warp == EPI_WARP0 && lane == 0) {
                        atomicAdd(&att->n_pairs, (unsigned long long)UM_TC * UM_TW);
                        int alive = 0;
                        for (int c = 0; c < UM_TC; ++c) alive += !S.dead[c];
                        atomicAdd(&att->n_live, (unsigned long long)S.tile_live * UM_TW);
                        S.tile_live = alive;
                        if (!alive) S.item_dead = 1;
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&S.acc_empty[s]);
                    mbar_arrive(&S.wd_empty);
                }
            }
            // fold the running maxima (8 shifts per candidate)
            float v = rmax;
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            if (rowok && (lane & 7) == 0 && v > -INFINITY) atomicMax(&S.rmax[cidx], f2ord(v));
        }
        __syncthreads();
        // ---- phase bookkeeping (every thread, same numbers)
        {
            const int tok = S.tok;                 // slice index of the end token, or -1
            const int nb = tok >= 0 ? tok + 1 : T; // full_b / mma_done phases
            const int nw = tok >= 0 ? tok : T;     // wd_full phases
            const int ne = tok >= 0 ? tok - 1 : T; // acc_empty / wd_empty arrivals (tok >= 1)
            for (int s = 0; s < 2; ++s) {
                const uint32_t cb = (uint32_t)((nb + 1 - s) >> 1);
                const uint32_t ce = (uint32_t)((ne + 1 - s) >> 1);
                ph.full[s] += cb;
                ph.done[s] += cb;
                ph.acc[s] += ce;
            }
            ph.wdf += (uint32_t)nw;
            ph.wde += (uint32_t)ne;
        }
        if (threadIdx.x < UM_TC && tile * UM_TC + threadIdx.x < C &&
            S.rmax[threadIdx.x] != f2ord(-INFINITY))
            atomicMax(rho_max + S.cp[threadIdx.x], S.rmax[threadIdx.x]);
        __syncthreads();
        if (S.abort) break;
    }
    if (S.abort) {
        if (threadIdx.x == 0) {
            atomicExch(&att->status, 3);
            if (mma_issued) { // let the MMAs in flight finish before TMEM goes away
                umma_commit(&S.drain);
                mbar_wait_bounded(&S.drain, 0u, kDrainCycles);
            }
        }
        // bulk copies in flight complete on their barriers: wait (bounded) for
        // the last phase the loader issued on each before the shared memory goes
        // away (a phase it never issued is not waited for)
        if (threadIdx.x == 32) {
            for (int s = 0; s < 2; ++s)
                if (S.last_full[s] >= 0)
                    mbar_wait_bounded(&S.full_b[s], par((uint32_t)S.last_full[s]), kDrainCycles);
            if (S.last_wd >= 0) mbar_wait_bounded(&S.wd_full, par((uint32_t)S.last_wd), kDrainCycles);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u)
                     : "memory");
}

} // namespace

bool paddi_umma_supported(int device)
{
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return p.major == 10 && p.minor == 0; // sm_100 (B200)
}

int paddi_umma_max_m() { return UM_KMAX64 - 7; } // kpad_of(m) <= UM_KMAX64

int32_t paddi_tile_width() { return UM_TW; }

int64_t paddi_tile_blocks(int64_t N) { return (N + UM_TW - 1) / UM_TW; }

int64_t paddi_tile_block_elems_max() { return 2 * (int64_t)slice_cnt(UM_KMAX64); }

int64_t paddi_tile_wd_entries() { return (int64_t)8 * WD_ROW; }

PaddiBound paddi_bound_tc(int m, bool bf16)
{
    const double u = std::ldexp(1.0, -24);
    const int kp = kpad_of(m);
    // split representation: z and y each within 2^-22 (FP16) / 2^-16 (BF16) of
    // their value, the dropped lo*lo term as much again; FP16 z halves below the
    // normal range: 2^-25 absolute against |z| = 2^8, i.e. 2^-33 sqrt(m) relative
    const double rep = bf16 ? 3.0 * std::ldexp(1.0, -16)
                            : 3.0 * std::ldexp(1.0, -22) + std::ldexp(1.0, -33) * std::sqrt((double)m);
    // the accumulator: one FP32 rounding (taken as 2^-23, truncation) of at most
    // the sum of |products| per MMA, 3 kp/16 MMAs plus the block sums
    const double acc = std::ldexp(1.0, -23) * (3.0 * kp / 16.0 + 1.0);
    // the candidate's split-value sum (2 kp/16 terms per thread + 4 shuffle
    // levels), its z (two-float centring, scale: 4u), the slice's x - s (u), the
    // epilogue's a, b and FMA (4u), the FP32 rounding of thr (2u)
    const double rest = (2.0 * kp / 16.0 + 4.0 + 4.0 + 1.0 + 4.0 + 2.0) * u; // + thr's rounding
    PaddiBound B;
    B.E = (float)((rep + acc + rest) * 1.01);
    // FP16 y halves below the normal range: 2^-25 per scaled value, 2^-(8+e) <=
    // 2 |x - s|_max 2^-22 of scale, against |z| sqrt(m) 2^8: 2^-38 sqrt(m) |x - s|_max
    B.F = bf16 ? 0.f : (float)(std::ldexp(1.0, -38) * std::sqrt((double)m) * 1.01);
    return B;
}

cudaError_t paddi_launch_tile_prep(bool bf16, const float *x, int64_t n, int32_t m,
                                   const float4 *wst, const float *mu, uint16_t *bq, float4 *wdq,
                                   float gcap, int32_t *frag_list, int32_t *frag_count,
                                   cudaStream_t st)
{
    const int kp = kpad_of(m);
    if (kp > UM_KMAX64 || m < 3) return cudaErrorInvalidValue;
    const int64_t N = n - m + 1;
    const unsigned grid = (unsigned)paddi_tile_blocks(N);
    const PaddiBound B = paddi_bound_tc(m, bf16);
    if (bf16)
        k_tile_prep<true><<<grid, TP_THREADS, 0, st>>>(x, n, slice_cnt(kp), m, wst, mu, bq, wdq,
                                                       B.E, B.F, gcap, frag_list, frag_count);
    else
        k_tile_prep<false><<<grid, TP_THREADS, 0, st>>>(x, n, slice_cnt(kp), m, wst, mu, bq, wdq,
                                                        B.E, B.F, gcap, frag_list, frag_count);
    return cudaGetLastError();
}

cudaError_t paddi_launch_refine_umma(bool bf16, const float *x, const float4 *wst,
                                     const float *mu, const int32_t *cand, const int32_t *list,
                                     const int32_t *list_count, const uint16_t *bq,
                                     const float4 *wdq, PaddiAttemptDev *att, int32_t *work,
                                     uint32_t *rho_max, uint8_t *pruned, int32_t N, int32_t m,
                                     int32_t jb, int32_t je, float thr_prune, int32_t num_sms,
                                     cudaStream_t st, long long wait_cycles, int32_t withhold,
                                     int32_t round, int32_t je_all, bool rows64)
{
    const int kp = kpad_of(m);
    if (kp > UM_KMAX64 || m < 3) return cudaErrorInvalidValue;
    if ((jb % UM_TW) != 0 || (je % UM_TW != 0 && je != N)) return cudaErrorInvalidValue;
    if (je_all > 0 && (je_all < je || (je_all % UM_TW != 0 && je_all != N)))
        return cudaErrorInvalidValue;
    const int MM = (kp <= UM_KMAX128 && !rows64) ? 128 : 64;
    const UmLayout L = um_layout(MM, kp);
    // request at least half the SM's shared memory so one CTA owns the 512 TMEM columns
    const size_t smem = L.bytes < 120 * 1024 ? 120 * 1024 : L.bytes;
    void (*kern)(const float *, const float4 *, const float *, const int32_t *, const int32_t *,
                 const int32_t *, const uint16_t *, const float4 *, PaddiAttemptDev *, int32_t *,
                 uint32_t *, uint8_t *, int32_t, int32_t, int32_t, int32_t, float, int32_t,
                 long long, int32_t, int32_t, int32_t);
    if (MM == 128) kern = bf16 ? k_refine_umma<true, 128> : k_refine_umma<false, 128>;
    else kern = bf16 ? k_refine_umma<true, 64> : k_refine_umma<false, 64>;
    cudaError_t e = paddi_raise_smem_limit((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    const int grid = num_sms;
    kern<<<grid, UM_THREADS, smem, st>>>(x, wst, mu, cand, list, list_count, bq, wdq, att, work,
                                         rho_max, pruned, N, m, jb, je, thr_prune, grid,
                                         wait_cycles > 0 ? wait_cycles : 4000000000ll, withhold,
                                         round, je_all > 0 ? je_all : je);
    return cudaGetLastError();
}
