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
// Pipeline per CTA (one CTA per SM, 512 TMEM columns = two 128x256 FP32
// accumulators): while the tensor core computes tile t+1 into one
// accumulator, the 8 warps convert the slice of tile t+2 into the free
// shared-memory stage and run the epilogue of tile t from the other
// accumulator (tcgen05.ld, distance, exclusion, running max, prune flags).
// Every mbarrier wait is bounded; on timeout the kernel records status 3,
// releases its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <float.h>

#include "paddi_internal.cuh"

using paddi::f2ord;

namespace {

constexpr int UM_THREADS = 256;  // 8 warps
constexpr int UM_TCMAX = 16;     // candidates per tile (M = 128); 8 for M = 64
constexpr int UM_N = 256;        // windows at stride 8
constexpr int UM_TW = UM_N * 8;  // windows per tile
constexpr int UM_KMAX128 = 368;  // largest K' with M = 128 (shared-memory bound)
constexpr int UM_KMAX64 = 736;   // largest K' with M = 64
constexpr int ZSCALE = 8;        // zhat scaled by 2^8 before splitting
constexpr long long UM_WAIT_CYCLES = 4000000000ll; // ~2 s at 1.9 GHz

__host__ __device__ constexpr int kpad_of(int m) { return ((m + 7) + 15) & ~15; }

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

// Bounded wait; false when the limit was reached.
__device__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > UM_WAIT_CYCLES) return false;
    return true;
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

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
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
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
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

// ------------------------------------------------------------------ shared memory
struct UmLayout {
    uint32_t a_hi, a_lo, b[2][2], wd, bytes;
};

__host__ __device__ inline UmLayout um_layout(int MM, int kp)
{
    UmLayout L;
    const uint32_t a_bytes = (uint32_t)MM * kp * 2;
    const uint32_t b_bytes = ((uint32_t)(UM_TW + kp + 16) * 2 + 127) & ~127u;
    L.a_hi = 0;
    L.a_lo = a_bytes;
    uint32_t o = 2 * a_bytes;
    for (int s = 0; s < 2; ++s)
        for (int h = 0; h < 2; ++h) {
            L.b[s][h] = o;
            o += b_bytes;
        }
    L.wd = o; // float2 (mu, inv) per window of the current tile
    o += UM_TW * 8;
    L.bytes = o;
    return L;
}

struct UmShared {
    uint64_t mbar[2];
    uint32_t tmem_base;
    int item, abort, alive;
    float sh[3];     // shift of the tile held by each stage (and the next one)
    float dscale[3]; // 2^-(ZSCALE + e) of the tile
    int cw[UM_TCMAX], cp[UM_TCMAX];
    float cflat[UM_TCMAX], zsum[UM_TCMAX];
    uint32_t rmax[UM_TCMAX];
    uint8_t dead[UM_TCMAX];
};

// Converts the slice of the tile starting at window j0 into stage buffers.
// One global read per value: the values stay in registers between the
// magnitude reduction and the split (at most CV_PER values per thread).
constexpr int CV_PER = (UM_TW + UM_KMAX64 + 16 + UM_THREADS - 1) / UM_THREADS;

template <bool BF>
__device__ void um_convert(unsigned char *smem, const UmLayout &L, int stage, const float *x,
                           int64_t nser, int j0, int kp, float *sh_out, float *dscale_out,
                           float *red)
{
    using X = E16<BF>;
    typename X::T *hi = reinterpret_cast<typename X::T *>(smem + L.b[stage][0]);
    typename X::T *lo = reinterpret_cast<typename X::T *>(smem + L.b[stage][1]);
    const int cnt = UM_TW + kp + 16;
    const float sh = __ldg(x + j0);
    float v[CV_PER];
    float mx = 0.f;
#pragma unroll
    for (int i = 0; i < CV_PER; ++i) {
        const int p = threadIdx.x + i * UM_THREADS;
        const int64_t g = (int64_t)j0 + p;
        v[i] = (p < cnt && g < nser) ? __ldg(x + g) - sh : 0.f;
        mx = fmaxf(mx, fabsf(v[i]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    mx = 0.f;
#pragma unroll
    for (int w = 0; w < UM_THREADS / 32; ++w) mx = fmaxf(mx, red[w]);
    int e = 0;
    if (mx > 0.f) {
        int ex;
        frexpf(mx, &ex); // mx = f * 2^ex, f in [0.5, 1)
        e = 14 - ex;     // mx * 2^e < 2^14
        e = max(-100, min(100, e));
    }
    const float sc = ldexpf(1.f, e);
#pragma unroll
    for (int i = 0; i < CV_PER; ++i) {
        const int p = threadIdx.x + i * UM_THREADS;
        if (p < cnt) {
            const float u = v[i] * sc;
            const typename X::T h = X::cvt(u);
            hi[p] = h;
            lo[p] = X::cvt(u - X::back(h));
        }
    }
    if (threadIdx.x == 0) {
        *sh_out = sh;
        *dscale_out = ldexpf(1.f, -(ZSCALE + e));
    }
}

// MM = 128: 16 candidates, accumulator row r in TMEM lane r.
// MM = 64:  8 candidates, accumulator row r in TMEM lane (r % 16) + 32 (r / 16)
//           (lanes 16..31 of every subpartition stay unused).
template <bool BF, int MM>
__global__ void __launch_bounds__(UM_THREADS, 1)
k_refine_umma(const float *__restrict__ x, const float4 *__restrict__ wst,
              const float *__restrict__ mu, const int32_t *__restrict__ cand,
              const int32_t *__restrict__ list, const int32_t *__restrict__ list_count,
              PaddiAttemptDev *att, uint32_t *rho_max, uint8_t *pruned, int32_t N, int32_t m,
              int32_t jb, int32_t je, float thr, int32_t grid_ctas)
{
    using X = E16<BF>;
    constexpr int UM_M = MM;
    constexpr int UM_TC = MM / 8;
    constexpr int RG = MM / 8;          // 8-row core-matrix groups of A
    extern __shared__ __align__(1024) unsigned char um_smem[];
    __shared__ UmShared S;
    __shared__ float red[UM_THREADS / 32];
    const int kp = kpad_of(m);
    const UmLayout L = um_layout(MM, kp);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nser = (int64_t)N + m - 1;

    const int C = *list_count;
    if (C <= 0 || je <= jb) return; // uniform: before any TMEM or barrier use

    if (threadIdx.x == 0) {
        mbar_init(&S.mbar[0], 1);
        mbar_init(&S.mbar[1], 1);
        S.abort = 0;
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
    uint32_t waits0 = 0u, waits1 = 0u; // completed waits per accumulator (parity source)

    const int range = je - jb;
    const int tiles = (C + UM_TC - 1) / UM_TC;
    int splits = (2 * grid_ctas + tiles - 1) / tiles;
    splits = max(1, min(splits, max(1, range / (2 * UM_TW))));
    const int span = (((range + splits - 1) / splits) + UM_TW - 1) / UM_TW * UM_TW;
    const int total = tiles * splits;
    const uint32_t idesc = idesc_f16(X::fmt, UM_M, UM_N);
    const uint32_t a_hi_s = smem_u32(um_smem + L.a_hi), a_lo_s = smem_u32(um_smem + L.a_lo);
    const int kblocks = kp / 16;
    // epilogue geometry: lane group g (TMEM lanes 32g..32g+31), column half h
    const int g = warp & 3, hcol = warp >> 2;
    const bool rowok = MM == 128 || lane < 16;
    const int row = MM == 128 ? 32 * g + lane : 16 * g + (lane & 15);
    const int cidx = row >> 3, bsh = row & 7;

    for (;;) {
        if (threadIdx.x == 0) S.item = atomicAdd(&att->work_next, 1);
        __syncthreads();
        const int item = S.item;
        if (item >= total || S.abort) break;
        const int tile = item % tiles, split = item / tiles;
        const int j_lo = jb + split * span, j_hi = min(je, j_lo + span);
        if (j_lo >= j_hi) { // empty split (all threads agree); keep S.item stable
            __syncthreads();
            continue;
        }
        if (threadIdx.x < UM_TC) {
            const int li = tile * UM_TC + threadIdx.x;
            const bool v = li < C;
            const int pos = v ? list[li] : 0;
            const int w = v ? cand[pos] : 0;
            S.cw[threadIdx.x] = w;
            S.cp[threadIdx.x] = pos;
            S.dead[threadIdx.x] = !v || __ldcg(pruned + pos);
            S.cflat[threadIdx.x] = v ? wst[w].w : 0.f;
            S.rmax[threadIdx.x] = f2ord(-INFINITY);
        }
        __syncthreads();
        {
            int a = threadIdx.x < UM_TC ? !S.dead[threadIdx.x] : 0;
            if (!__syncthreads_or(a)) continue;
        }
        // ---- candidate operand: 16 x (hi, lo) rows of scaled zhat, then 8 shifted copies
        {
            typename X::T *zh = reinterpret_cast<typename X::T *>(um_smem + L.b[0][0]);
            typename X::T *zl = zh + UM_TC * kp; // aliases the stage buffers (idle here)
            const int c = threadIdx.x >> 4, t16 = threadIdx.x & 15;
            const int w = c < UM_TC ? S.cw[c] : 0;
            const bool live = c < UM_TC && !S.dead[c];
            const float muc = live ? mu[w] : 0.f;
            const float ivc = live ? wst[w].z * 256.f : 0.f; // 2^ZSCALE
            float zs = 0.f;
            for (int k = t16; k < kp; k += 16) {
                const float v = (live && k < m) ? (x[w + k] - muc) * ivc : 0.f;
                const typename X::T h = X::cvt(v);
                const typename X::T l = X::cvt(v - X::back(h));
                if (c < UM_TC) {
                    zh[c * kp + k] = h;
                    zl[c * kp + k] = l;
                }
                zs += X::back(h) + X::back(l);
            }
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) zs += __shfl_xor_sync(0xffffffffu, zs, o);
            if (t16 == 0 && c < UM_TC) S.zsum[c] = zs * (1.f / 256.f);
            __syncthreads();
            // A[(c,b), k'] = z_c[k' - b] in K-major core matrices:
            // byte offset ((k'/8)*RG + r/8)*128 + (r%8)*16 + (k'%8)*2
            const int chunks = kp / 8;
            for (int e = threadIdx.x; e < UM_M * chunks; e += UM_THREADS) {
                const int r = e & (UM_M - 1), kc = e / UM_M;
                const int cc = r >> 3, b = r & 7;
                uint32_t ph[4], pl[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int k0 = kc * 8 + 2 * q - b, k1 = k0 + 1;
                    typename X::T h0 = X::cvt(0.f), h1 = X::cvt(0.f), l0 = X::cvt(0.f),
                                  l1 = X::cvt(0.f);
                    if (k0 >= 0 && k0 < kp) {
                        h0 = zh[cc * kp + k0];
                        l0 = zl[cc * kp + k0];
                    }
                    if (k1 >= 0 && k1 < kp) {
                        h1 = zh[cc * kp + k1];
                        l1 = zl[cc * kp + k1];
                    }
                    ph[q] = (uint32_t)reinterpret_cast<uint16_t &>(h0) |
                            ((uint32_t)reinterpret_cast<uint16_t &>(h1) << 16);
                    pl[q] = (uint32_t)reinterpret_cast<uint16_t &>(l0) |
                            ((uint32_t)reinterpret_cast<uint16_t &>(l1) << 16);
                }
                const uint32_t off = (uint32_t)((kc * RG + (r >> 3)) * 128 + (r & 7) * 16);
                *reinterpret_cast<uint4 *>(um_smem + L.a_hi + off) =
                    make_uint4(ph[0], ph[1], ph[2], ph[3]);
                *reinterpret_cast<uint4 *>(um_smem + L.a_lo + off) =
                    make_uint4(pl[0], pl[1], pl[2], pl[3]);
            }
            __syncthreads(); // zh/zl reads done before the stages are overwritten
        }
        // ---- tile pipeline
        const int T = (j_hi - j_lo + UM_TW - 1) / UM_TW;
        um_convert<BF>(um_smem, L, 0, x, nser, j_lo, kp, &S.sh[0], &S.dscale[0], red);
        fence_proxy_async_smem();
        __syncthreads();
        auto issue = [&](int t) { // tile t -> accumulator t&1 from stage t&1
            const int s = t & 1;
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
            umma_commit(&S.mbar[s]);
        };
        if (threadIdx.x == 0) {
            tc_fence_after();
            issue(0);
        }
        float tsh0 = S.sh[0], tds0 = S.dscale[0], tsh1 = 0.f, tds1 = 0.f;
        if (T > 1) {
            __syncthreads(); // S.sh[0] read before it is rewritten
            um_convert<BF>(um_smem, L, 1, x, nser, j_lo + UM_TW, kp, &S.sh[1], &S.dscale[1], red);
            fence_proxy_async_smem();
        }
        __syncthreads();
        if (T > 1) {
            tsh1 = S.sh[1];
            tds1 = S.dscale[1];
        }
        float rmax = -INFINITY;
        const int wc = S.cw[cidx];
        const float zsc = S.zsum[cidx], fc = S.cflat[cidx];
        for (int t = 0; t < T; ++t) {
            const int s = t & 1;
            const int j0 = j_lo + t * UM_TW;
            if (t + 1 < T && threadIdx.x == 0) {
                tc_fence_after();
                issue(t + 1); // overlaps with the work below
            }
            // wait for tile t
            if (threadIdx.x == 0) {
                if (!mbar_wait_bounded(&S.mbar[s], (s ? waits1 : waits0) & 1u)) S.abort = 1;
            }
            __syncthreads();
            if (s) ++waits1;
            else ++waits0;
            if (S.abort) break;
            tc_fence_after();
            const float sh = s ? tsh1 : tsh0, dsc = s ? tds1 : tds0;
            // slice of tile t+2 into the stage tile t used (its MMAs are complete)
            if (t + 2 < T) {
                um_convert<BF>(um_smem, L, s, x, nser, j0 + 2 * UM_TW, kp, &S.sh[2], &S.dscale[2],
                               red);
                fence_proxy_async_smem();
            }
            // per window of tile t: (inv * dscale, (mu - shift) * inv), so that
            // rho = D * wd.x - zsum_c * wd.y (+1 for two flat windows)
            float2 *wd = reinterpret_cast<float2 *>(um_smem + L.wd);
            {
                float mv[UM_TW / UM_THREADS], iv[UM_TW / UM_THREADS];
#pragma unroll
                for (int i = 0; i < UM_TW / UM_THREADS; ++i) {
                    const int q = threadIdx.x + i * UM_THREADS;
                    mv[i] = __ldg(mu + j0 + q);    // padded tail is zero
                    iv[i] = __ldg(&wst[j0 + q].z);
                }
#pragma unroll
                for (int i = 0; i < UM_TW / UM_THREADS; ++i)
                    wd[threadIdx.x + i * UM_THREADS] = make_float2(iv[i] * dsc, (mv[i] - sh) * iv[i]);
            }
            __syncthreads();
            // ---- epilogue: 128 columns per thread; a thread needs the
            // exclusion / range mask only when its candidate's trivial-match
            // zone or the end of the item range reaches into the tile
            const uint32_t tb = tmem + ((uint32_t)(32 * g) << 16) + (uint32_t)(s * UM_N + 128 * hcol);
            const bool masked = (j0 + UM_TW > j_hi) || (wc > j0 - m + 1 && wc < j0 + UM_TW + m - 1);
            float tmax = -INFINITY;
#pragma unroll 1
            for (int cb = 0; cb < 4; ++cb) {
                uint32_t r[32];
                tmem_ld32(tb + 32 * cb, r);
                const int qb = 8 * (128 * hcol + 32 * cb) + bsh;
                if (!masked && fc == 0.f) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const float2 wv = wd[qb + 8 * i];
                        tmax = fmaxf(tmax, fmaf(__uint_as_float(r[i]), wv.x, -zsc * wv.y));
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const int q = qb + 8 * i, j = j0 + q;
                        const float2 wv = wd[q];
                        float rho = fmaf(__uint_as_float(r[i]), wv.x, -zsc * wv.y);
                        if (fc != 0.f && wv.x == 0.f) rho += 1.f; // two flat windows
                        const int dd = wc > j ? wc - j : j - wc;
                        if (j < j_hi && dd >= m - 1) tmax = fmaxf(tmax, rho);
                    }
                }
            }
            if (!rowok) tmax = -INFINITY;
            rmax = fmaxf(rmax, tmax);
            const bool hit = tmax > thr;
            tc_fence_before();
            const unsigned bal = __ballot_sync(0xffffffffu, hit);
            if (lane < UM_TC / 4 && ((bal >> (8 * lane)) & 0xFFu)) {
                const int ci = (UM_TC / 4) * g + lane;
                if (!S.dead[ci]) {
                    S.dead[ci] = 1;
                    pruned[S.cp[ci]] = 1;
                }
            }
            if (threadIdx.x == 0)
                atomicAdd(&att->n_pairs, (unsigned long long)UM_TC * UM_TW);
            __syncthreads();
            if (t + 2 < T) { // stage parameters of tile t+2
                if (s) {
                    tsh1 = S.sh[2];
                    tds1 = S.dscale[2];
                } else {
                    tsh0 = S.sh[2];
                    tds0 = S.dscale[2];
                }
            }
            // early abandoning: stop once every candidate of the tile is pruned
            int alive_c = 0;
            if (threadIdx.x < UM_TC && !S.dead[threadIdx.x]) {
                if (__ldcg(pruned + S.cp[threadIdx.x])) S.dead[threadIdx.x] = 1;
                else alive_c = 1;
            }
            if (!__syncthreads_or(alive_c)) {
                if (t + 1 < T) { // drain the MMAs of tile t+1 before leaving the item
                    const int s1 = (t + 1) & 1;
                    if (threadIdx.x == 0 &&
                        !mbar_wait_bounded(&S.mbar[s1], (s1 ? waits1 : waits0) & 1u))
                        S.abort = 1;
                    __syncthreads();
                    if (s1) ++waits1;
                    else ++waits0;
                }
                break;
            }
        }
        // ---- fold the running maxima (8 shifts x 2 column halves per candidate)
        float v = rmax;
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (rowok && (lane & 7) == 0 && v > -INFINITY) atomicMax(&S.rmax[cidx], f2ord(v));
        __syncthreads();
        if (threadIdx.x < UM_TC && tile * UM_TC + threadIdx.x < C &&
            S.rmax[threadIdx.x] != f2ord(-INFINITY))
            atomicMax(rho_max + S.cp[threadIdx.x], S.rmax[threadIdx.x]);
        __syncthreads();
        if (S.abort) break;
    }
    if (S.abort && threadIdx.x == 0) atomicExch(&att->status, 3);
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

cudaError_t paddi_launch_refine_umma(bool bf16, const float *x, const float4 *wst,
                                     const float *mu, const int32_t *cand, const int32_t *list,
                                     const int32_t *list_count, PaddiAttemptDev *att,
                                     uint32_t *rho_max, uint8_t *pruned, int32_t N, int32_t m,
                                     int32_t jb, int32_t je, float thr_prune, int32_t num_sms,
                                     cudaStream_t st)
{
    const int kp = kpad_of(m);
    if (kp > UM_KMAX64 || m < 3) return cudaErrorInvalidValue;
    const int MM = kp <= UM_KMAX128 ? 128 : 64;
    const UmLayout L = um_layout(MM, kp);
    // request at least half the SM's shared memory so one CTA owns the 512 TMEM columns
    const size_t smem = L.bytes < 120 * 1024 ? 120 * 1024 : L.bytes;
    void (*kern)(const float *, const float4 *, const float *, const int32_t *, const int32_t *,
                 const int32_t *, PaddiAttemptDev *, uint32_t *, uint8_t *, int32_t, int32_t,
                 int32_t, int32_t, float, int32_t);
    if (MM == 128) kern = bf16 ? k_refine_umma<true, 128> : k_refine_umma<false, 128>;
    else kern = bf16 ? k_refine_umma<true, 64> : k_refine_umma<false, 64>;
    cudaError_t e = paddi_raise_smem_limit((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    const int grid = num_sms;
    kern<<<grid, UM_THREADS, smem, st>>>(x, wst, mu, cand, list, list_count, att, rho_max, pruned,
                                         N, m, jb, je, thr_prune, grid);
    return cudaGetLastError();
}
