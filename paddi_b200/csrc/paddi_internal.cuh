// paddi_internal.cuh -- shared device helpers and launch wrappers of the
// discord-discovery kernels (single GPU, sm_100a).
//
// Per-window data for one subsequence length m, laid out in HBM as arrays
// over the N = n - m + 1 windows (plus PADDI_PAD_WIN zeroed entries so tiles
// may read past the end without bounds checks):
//   wst[i]  float4 {df_i, dg_i, inv_i, n_i}   -- diagonal-update terms
//           df_i = (x[i+m] - x[i]) / 2,  dg_i = (x[i+m] - mu_{i+1}) + (x[i] - mu_i)
//           n_i = |x_i - mu_i| (the window's norm), inv_i = 1 / n_i; both 0 for
//           a flat window (window i is flat iff inv_i == 0)
//   mu[i]   float  window mean
//   mu64[i], inv64[i]  FP64 mean and inverse norm (recheck path)
//   flat[i] uint8
// The correlation of windows i, j is rho = cov(i,j) * inv_i * inv_j with
// cov the centred dot product; the squared z-normalised distance is
// d = 2m (1 - rho) (reference: src/PD3_kernels.cuh:61).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

/* zeroed tail entries after the last window: covers the columns a phase-1
 * task of up to 4096 rows reads past the end (rows + 256) and a tile of the
 * tensor-core refine (2048 windows) */
#define PADDI_PAD_WIN 4608

namespace paddi {

// Monotone map float -> uint32 so that unsigned max == float max.
__device__ __forceinline__ uint32_t f2ord(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}
// Monotone map double -> uint64 (for FP64 atomic min/max).
__device__ __forceinline__ unsigned long long d2ord(double d)
{
    unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord2d(unsigned long long u)
{
    return __longlong_as_double((long long)((u & 0x8000000000000000ull)
                                                ? (u & 0x7fffffffffffffffull)
                                                : ~u));
}

// Rounding bound, in correlation units, of a refine kernel's correlation of
// any candidate with window j whose operand is the series shifted by s:
//     g_j = E * A_j + F * inv_j,   A_j = |x_j - s| / |x_j - mu_j| = sqrt(1 + m b^2),
// b = (mu_j - s) inv_j.  E (per kernel and length) bounds the relative error of
// the dot product with respect to |z| |x_j - s| (|z| = 1), F an absolute error
// term of the operand's representation.  Explicitly rounded operations, so
// every kernel that evaluates it for the same window gets the same value.
__device__ __forceinline__ float window_bound(float inv, float mu, float s, float m, float E,
                                              float F)
{
    const float b = __fmul_rn(__fsub_rn(mu, s), inv);
    const float A = __fsqrt_rn(__fadd_rn(1.f, __fmul_rn(m, __fmul_rn(b, b))));
    return __fadd_rn(__fmul_rn(__fmul_rn(E, A), 1.0001f), __fmul_rn(F, inv));
}

} // namespace paddi

// Bound constants of the refine kernels for length m (see window_bound):
// E covers the 16-bit split operands (FP16: 2^-22 per value and the dropped
// lo*lo term; BF16: 2^-16), one FP32 rounding per tensor-core MMA of the
// accumulator (3 kp/16 MMAs, kp = K padded) and the FP32 arithmetic around it
// (the candidate's z, the sum of its split values, the epilogue); F covers
// FP16 lo halves that fall below the normal range (2^-25 absolute per scaled
// value; F is per unit of the tile's largest |x - s|).  The FP32 CUDA-core
// refine sums in two levels of 32 terms and has F = 0.
struct PaddiBound {
    float E, F;
};
PaddiBound paddi_bound_tc(int m, bool bf16);
PaddiBound paddi_bound_fp32(int m);

// Per-attempt device-side state shared by the kernels of one (m, r) attempt.
struct PaddiAttemptDev {
    int32_t n_cand_p1;      // candidates after phase 1 (compacted list length)
    int32_t work_rd[4];     // work-item counters of the refine rounds (one per round)
    int32_t recheck_next;   // work-item counter of the FP64 recheck kernel
    int32_t n_recheck;      // windows queued for the FP64 recheck (at most its capacity)
    int32_t n_recheck_all;  // windows that needed it: above the capacity, the queue overflowed
    int32_t status;         // nonzero: a kernel hit an internal limit
    int32_t task_next;      // task counter of the phase-1 kernel
    int32_t list_count[5];  // candidate-list length entering each refine round (and after
                            // the last); zero when the attempt starts, so the compactions
                            // between rounds need no reset
    int32_t p1_walked;      // phase-1 tasks that walked their rows (instrumentation)
    int32_t covered_from;   // r + 1 when refine round r (one candidate tile left) took
                            // every remaining window; later rounds then have nothing to do
    unsigned long long n_pairs; // pairs evaluated by the refine (instrumentation)
    unsigned long long n_live;  // of those, pairs of candidates still unpruned at the tile's start
};

// Result of one attempt, copied to the host at the end of the attempt.
struct PaddiAttemptResult {
    int64_t n_cand;  // windows with nn >= r2 (never pruned)
    int64_t n_disc;  // windows with nn > r2
    int32_t n_sel;   // discords selected (<= top_k)
    int32_t n_recheck;
    int32_t n_p1;    // candidates after phase 1
    int32_t status;
    int32_t sel_ind[16];
    float sel_dist[16];
    unsigned long long n_pairs; // refine pairs evaluated
    unsigned long long n_live;  // of those, pairs of candidates live at the tile's start
    int32_t p1_walked;          // phase-1 tasks that walked their rows
    int32_t n_fragile;          // windows the refine left to the FP64 fragile pass
};

// Incremental FP64 nn of the r policy's bound window (k_guide.cu): the state
// of the shifted dot products G (two buffers), the launch's result, and
// kernel counters.  A zeroed record holds no state (no length is 0).
enum { PADDI_GUIDE_SKIPPED = 0, PADDI_GUIDE_REUSED = 1, PADDI_GUIDE_SLID = 2,
       PADDI_GUIDE_BUILT = 3 };
struct PaddiGuide {
    unsigned long long nn_ord; // result: ordered image of the nn (all ones: none)
    double s;                  // state: shift of both operands of G
    int32_t w, m;              // state: window and length G holds
    int32_t cur, age;          // state: buffer holding G, slides since the last build
    int32_t w_used, mode;      // result: window of the launch (-1: skipped), PADDI_GUIDE_*
    int32_t done, item;        // kernel counters (zero between launches)
};

#define PADDI_MAX_TOPK 16
#define PADDI_MAX_RECHECK 1024 /* initial FP64 recheck capacity (grows on demand) */

// ---------------------------------------------------------------- launches
// All launch wrappers enqueue on `st` and return cudaGetLastError().
cudaError_t paddi_launch_stats(const float *x, int64_t n, int32_t m, float4 *wst, float *mu,
                               double *mu64, double *inv64, uint8_t *flat,
                               int32_t *flat_count, cudaStream_t st,
                               int32_t *flat_span = nullptr);
// flat_span (optional): two zeroed ints that receive {INT_MAX - lowest flat
// window, highest flat window + 1} (both stay 0 without flat windows).

// Phase 1 at threshold thr = 1 - r^2 / (2m): an exact test (the kernel bounds
// its own FP32 rounding, no guard band).
// Only the rows [row_lo, row_hi) are walked (their columns reach anywhere).
cudaError_t paddi_launch_phase1_dev(const float *x, const float4 *wst, const float *mu,
                                    const double *mu64, uint8_t *alive, int32_t N, int32_t m,
                                    int32_t R, int32_t max_chunks, float thr, int32_t row_lo,
                                    int32_t row_hi, int32_t *task_counter, int32_t *walked,
                                    int32_t num_sms, cudaStream_t st);

// prune_flats (r^2 > 0): flat windows with another flat window at least m-1
// away are dropped (distance 0); flat_span as filled by paddi_launch_stats.
cudaError_t paddi_launch_compact(const uint8_t *alive, int32_t N, int32_t *cand,
                                 uint32_t *rho_max, uint8_t *pruned, int32_t *rc_slot,
                                 PaddiAttemptDev *att, const uint8_t *flat,
                                 const int32_t *flat_span, int32_t m, bool prune_flats,
                                 cudaStream_t st);

// Dense refine of the candidates in list[0..*list_count) (positions into
// cand[]) against the windows [jb, je) (jb a multiple of 256).  thr is the
// exact threshold 1 - r^2 / (2m): the kernel prunes on lower bounds of the
// correlations; gcap is the guard band (fragile windows are skipped).
cudaError_t paddi_launch_refine_fp32(const float *x, const float4 *wst, const float *mu,
                                     const int32_t *cand, const int32_t *list,
                                     const int32_t *list_count, PaddiAttemptDev *att,
                                     int32_t *work, uint32_t *rho_max, uint8_t *pruned,
                                     int32_t N, int32_t m, int32_t jb, int32_t je, float thr,
                                     float gcap, int32_t num_sms, cudaStream_t st);

// Fragile windows of length m in the FP32 refine's geometry, appended to
// frag_list (frag_count zeroed by the caller).
cudaError_t paddi_launch_fragile_scan_fp32(const float *x, const float4 *wst, const float *mu,
                                           int32_t N, int32_t m, float gcap, int32_t *frag_list,
                                           int32_t *frag_count, int32_t num_sms, cudaStream_t st);

// Exact FP64 correlations of the unpruned candidates of list[0..*list_count)
// with the fragile windows in [col_lo, col_hi) (k_fragile.cu): prunes and
// raises rho_max.
cudaError_t paddi_launch_fragile(const float *x, const double *mu64, const double *inv64,
                                 const int32_t *cand, const int32_t *list,
                                 const int32_t *list_count, uint8_t *pruned, uint32_t *rho_max,
                                 const int32_t *frag, const int32_t *frag_count, int32_t m,
                                 float thr, int32_t col_lo, int32_t col_hi, int32_t num_sms,
                                 cudaStream_t st);

// Tensor-core refine over windows [jb, je) (jb a multiple of the tile width,
// je too or je = N).  bq / wdq: the per-length tile data of
// paddi_launch_tile_prep.  wait_cycles: limit of every barrier wait (<= 0:
// about 2 s); a wait that runs out sets att->status = 3 and the kernel
// returns.  withhold != 0 is a test hook: the CTA holding work item 0 never
// fills that item's first stage, so its waits run out.
cudaError_t paddi_launch_refine_umma(bool bf16, const float *x, const float4 *wst,
                                     const float *mu, const int32_t *cand, const int32_t *list,
                                     const int32_t *list_count, const uint16_t *bq,
                                     const float4 *wdq, PaddiAttemptDev *att, int32_t *work,
                                     uint32_t *rho_max, uint8_t *pruned, int32_t N, int32_t m,
                                     int32_t jb, int32_t je,
                                     float thr_prune, int32_t num_sms, cudaStream_t st,
                                     long long wait_cycles = 0, int32_t withhold = 0,
                                     int32_t round = 0, int32_t je_all = 0,
                                     bool rows64 = false);

// Per-length tile data of the tensor-core refine: for every block of
// paddi_tile_width() windows, the split 16-bit series slice (bq, at most
// paddi_tile_block_elems_max() elements per block) and the epilogue's window
// data (wdq, paddi_tile_wd_entries() float4 per block).
int32_t paddi_tile_width();
int64_t paddi_tile_blocks(int64_t N);
int64_t paddi_tile_block_elems_max();
int64_t paddi_tile_wd_entries();
// Fragile windows (bound above gcap) are appended to frag_list (frag_count
// zeroed by the caller).
cudaError_t paddi_launch_tile_prep(bool bf16, const float *x, int64_t n, int32_t m,
                                   const float4 *wst, const float *mu, uint16_t *bq, float4 *wdq,
                                   float gcap, int32_t *frag_list, int32_t *frag_count,
                                   cudaStream_t st);

cudaError_t paddi_launch_list_init(const PaddiAttemptDev *att, int32_t *list, int32_t *count,
                                   cudaStream_t st);

cudaError_t paddi_launch_list_compact(const int32_t *in, const int32_t *in_count,
                                      const uint8_t *pruned, int32_t *out, int32_t *out_count,
                                      cudaStream_t st);

cudaError_t paddi_launch_finalize(const int32_t *cand, PaddiAttemptDev *att,
                                  const uint32_t *rho_max, const uint8_t *pruned, int32_t m,
                                  float r2, float thr, float guard, float widen, int32_t top_k,
                                  const uint8_t *flat, int32_t rc_cap, int32_t *recheck,
                                  int32_t *rc_slot, unsigned long long *nn64_ord,
                                  PaddiAttemptResult *res, int32_t known_w,
                                  unsigned long long known_ord, cudaStream_t st);

cudaError_t paddi_launch_recheck(const float *x, const double *mu64, const double *inv64,
                                 const uint8_t *flat, int32_t N, int32_t m,
                                 const int32_t *cand, const int32_t *recheck,
                                 PaddiAttemptDev *att, unsigned long long *nn64_ord,
                                 int32_t num_sms, int32_t known_w, cudaStream_t st);

cudaError_t paddi_launch_select(const int32_t *cand, PaddiAttemptDev *att,
                                const uint32_t *rho_max, const uint8_t *pruned,
                                const int32_t *recheck, const int32_t *rc_slot,
                                const unsigned long long *nn64_ord, int32_t m, float r2,
                                float thr, float guard, int32_t top_k, const uint8_t *flat,
                                PaddiAttemptResult *res, cudaStream_t st);

// with_w: room for the flat-window column data (false only when the length is
// known to have no flat window).
size_t paddi_phase1_smem(int R, int m);

// Exact FP64 nn at length m of window w_host (w_host < 0: the top-1 window
// of the attempt result `prev`, skipped when it has none), through the shifted
// dot products (two buffers G of N doubles each, G + g_stride the second) and
// their state in g; result in g->nn_ord.
cudaError_t paddi_launch_guide(const float *x, const double *mu64, const double *inv64,
                               const uint8_t *flat, int32_t N, int32_t m,
                               const PaddiAttemptResult *prev, int32_t w_host, PaddiGuide *g,
                               double *G, size_t g_stride, int32_t num_sms, cudaStream_t st);

cudaError_t paddi_launch_export_stats(const double *mu64, const double *inv64, int32_t N,
                                      int32_t m, float *mean, float *sd, cudaStream_t st);

cudaError_t paddi_launch_scatter(const int32_t *cand, const PaddiAttemptDev *att,
                                 const uint32_t *rho_max, const uint8_t *pruned,
                                 const int32_t *rc_slot, const unsigned long long *nn64_ord,
                                 const uint8_t *flat, int32_t N, int32_t m, float r2,
                                 int32_t *is_cand, float *nnd, cudaStream_t st);

// Learned r predictor (k_mlp.cu).
#define MLP_NFEAT 12
#define MLP_HIDDEN 64
#define MLP_NPARAM (MLP_HIDDEN * MLP_NFEAT + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1)
cudaError_t paddi_launch_mlp_forward(const float *X, int n, const void *P, bool bf16, float *Y,
                                     cudaStream_t st);
cudaError_t paddi_launch_mlp_grad(const float *X, const float *Y, int n, float tau,
                                  const float *P, float *G, float *loss, int num_sms,
                                  cudaStream_t st);
cudaError_t paddi_launch_mlp_adam(float *P, float *G, float *M, float *V, float lr, int step,
                                  cudaStream_t st);
cudaError_t paddi_launch_mlp_to_bf16(const float *P, void *Q, cudaStream_t st);

// True when the tcgen05 split refine can run on `device`; longest m it takes.
// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device.  The limit is a process-wide attribute of the function, so
// host threads that launch the same kernel with different sizes could lower
// it under one another; here it only grows, under a lock.
cudaError_t paddi_raise_smem_limit(const void *func, size_t bytes);

bool paddi_umma_supported(int device);
int paddi_umma_max_m();
