/*
 * paddi.h -- C ABI of the B200 discord-discovery library (libpaddi.so).
 *
 * Drop-in for the per-GPU hot path of PADDi (KraevaYA/PADDi): PD3, the
 * DRAG-style fixed-length range-discord search, and PALMAD, the MERLIN-style
 * arbitrary-length search.  All entry points are plain C: pointers, sizes and
 * status codes, no C++ or framework types.
 *
 * Units and conventions follow the reference:
 *   - a discord is {start index, squared z-normalised distance to its
 *     nearest non-trivial neighbour}  (struct Discord, src/PALMAD_types.hpp:7-11);
 *   - the range threshold r is linear; kernels compare squared distances
 *     against r*r (src/main.cu:144 passes r*r);
 *   - windows i and j are trivial matches when |i - j| < m - 1
 *     (src/PD3_kernels.cuh:70);
 *   - a window is a candidate when no admissible neighbour is closer than
 *     r, a discord when its nearest-neighbour distance exceeds r
 *     (src/sets_processing.hpp:28-37); the top-1 is the first maximum.
 * Where the reference calls exit(1) on a CUDA error (src/common.h:6-16) these
 * functions return a status; paddi_last_error() gives the message.
 *
 * Threading: a context belongs to one host thread at a time and owns one
 * CUDA stream; use one context per thread for concurrency.
 */
#ifndef PADDI_H
#define PADDI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PADDI_ABI_VERSION 2

typedef enum paddi_status {
    PADDI_OK = 0,
    PADDI_ERR_INVALID_ARG = 1,  /* bad pointer, size or length range */
    PADDI_ERR_CUDA = 2,         /* a CUDA call failed (see paddi_last_error) */
    PADDI_ERR_OUT_OF_MEMORY = 3,
    PADDI_ERR_ITER_CAP = 4,     /* the r-schedule did not converge within iter_cap attempts */
    PADDI_ERR_NO_DEVICE = 5,    /* no CUDA device, or not an sm_100 device */
    PADDI_ERR_INTERNAL_LIMIT = 6, /* an internal capacity was exceeded */
    PADDI_ERR_UNSUPPORTED = 7   /* option value not supported by this build */
} paddi_status;

/* One discord.  Reference: struct Discord {int ind; float dist;} (src/PALMAD_types.hpp:7-11). */
typedef struct paddi_discord {
    int32_t ind;  /* start index of the window, -1 when none */
    float dist;   /* squared z-normalised nn distance, -FLT_MAX when none */
} paddi_discord;

/* Distance kernel for the dense candidate refine. */
typedef enum paddi_distance_kernel {
    PADDI_DIST_AUTO = 0,       /* split-FP16 tensor cores where the length allows, else FP32 */
    PADDI_DIST_FP32 = 1,       /* FP32 CUDA cores (the plain form) */
    PADDI_DIST_SPLIT_BF16 = 2, /* three-term BF16 split on tcgen05 tensor cores */
    PADDI_DIST_SPLIT_FP16 = 3  /* three-term FP16 split (scaled) on tcgen05 tensor cores */
} paddi_distance_kernel;

/* Where PALMAD's threshold for the next length comes from. */
typedef enum paddi_r_policy {
    PADDI_R_MERLIN = 0,   /* the reference schedule, src/main.cu:136-233 */
    PADDI_R_LEARNED = 1,  /* the bound where it is tight, else the learned predictor (paddi_model_*) */
    PADDI_R_BOUND = 2     /* first try r^2 just below the exact nn, at this length, of the
                             previous length's top-1 window (a lower bound on this
                             length's top-1 distance, so the try always succeeds);
                             MERLIN as fallback.  BOUND and LEARNED keep the bound's
                             FP64 dot products resident between lengths: the context
                             allocates 16 bytes per window on its first guided call */
} paddi_r_policy;

typedef struct paddi_opts {
    uint32_t struct_size;     /* sizeof(paddi_opts) */
    int32_t device;           /* CUDA device ordinal */
    int32_t distance_kernel;  /* paddi_distance_kernel */
    int32_t r_policy;         /* paddi_r_policy */
    uint32_t segment_len;     /* phase-1 rows per segment (reference SEGMENT_N); 0 = 256,
                                 else 64..4096 (others: PADDI_ERR_UNSUPPORTED) */
    uint32_t phase1_chunks;   /* 256-diagonal chunks a segment scans before the refine; 0 = 12 */
    uint32_t iter_cap;        /* attempts allowed per length; 0 = 200 */
    float guard;              /* guard band in correlation units: the largest per-window
                                 rounding bound the FP32 / split-16-bit refines accept (a
                                 window above it is evaluated in FP64) and the half-width
                                 of the FP64 recheck band; 0 = default (2e-4; 1e-3 for
                                 split-BF16) */
    uint32_t flags;           /* PADDI_FLAG_* */
    uint32_t tile_rows;       /* rows M of the tensor-core refine's tiles (8 shifts of M/8
                                 candidates): 0 = by length (128 while K' = m + 7 rounded
                                 to 16 is at most 368, else 64), 64 = always 64; others:
                                 PADDI_ERR_UNSUPPORTED.  Results do not depend on it. */
} paddi_opts;

/* paddi_opts.flags: compute the bound (paddi_attempt_log.lb) under every r
 * policy, e.g. to collect training features from plain MERLIN runs. */
#define PADDI_FLAG_LOG_BOUND 1u

/* One (length, r) attempt; the columns of the reference's times table
 * (src/IOdata.hpp:142-145) plus the values that drive the r-schedule. */
typedef struct paddi_attempt_log {
    int32_t m;            /* subsequence length */
    float r;              /* linear threshold */
    float r2;             /* r*r, the value the kernels compare against */
    int32_t found;        /* 1 when the attempt produced the requested discords */
    int64_t n_cand;       /* "# Candidates": windows never pruned (nn >= r2) */
    int64_t n_disc;       /* "# Discords": windows with nn > r2 */
    int64_t n_phase1;     /* candidates left after phase 1 */
    int32_t n_recheck;    /* windows whose distance was recomputed in FP64 */
    paddi_discord top;    /* best discord of the attempt */
    float ms_stats;       /* window statistics (once per length, logged on its first attempt) */
    float ms_phase1;      /* phase 1 */
    float ms_refine;      /* compaction + dense refine */
    float ms_select;      /* classification, FP64 recheck, top-k */
    float ms_total;       /* the whole attempt */
    int64_t refine_pairs; /* (candidate, window) pairs the dense refine evaluated */
    int32_t n_launches;   /* kernels this attempt launched (statistics included on its first) */
    int32_t refine_kernel; /* paddi_distance_kernel that ran the refine (1, 2 or 3) */
    int32_t r_source;     /* where r came from: 0 MERLIN schedule, 1 learned, 2 bound */
    float ms_guide;       /* time spent choosing r (bound / model), logged on the first attempt */
    float lb;             /* exact nn at this length of the previous length's top-1 window
                             (a lower bound on this length's top-1 distance); 0 if not computed */
    float flat_frac;      /* fraction of flat windows at this length */
    int64_t p1_pairs;     /* (row, diagonal) pairs phase 1 walked */
    int64_t refine_live_pairs; /* of refine_pairs, those whose candidate was still
                                  unpruned when its tile started */
    float ms_refine_kernel; /* the refine launches alone (ms_refine less the rounds'
                               candidate re-compaction) */
    int32_t n_fragile;    /* windows whose rounding bound in the refine exceeds the
                             guard band; their pairs were evaluated in FP64 */
} paddi_attempt_log;

typedef struct paddi_ctx paddi_ctx;

/* Library / context management. */
int32_t paddi_abi_version(void);
const char *paddi_status_string(paddi_status s);
void paddi_opts_default(paddi_opts *opts);
paddi_status paddi_ctx_create(paddi_ctx **ctx, const paddi_opts *opts);
paddi_status paddi_ctx_destroy(paddi_ctx *ctx);
const char *paddi_last_error(const paddi_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t): every kernel of the context
 * runs on it, so callers can order or time work against it. */
void *paddi_ctx_stream(paddi_ctx *ctx);
/* Reserve device memory for series of up to n values and lengths up to maxL
 * (optional: the entry points grow the reservation on demand). */
paddi_status paddi_ctx_reserve(paddi_ctx *ctx, size_t n, uint32_t maxL);

/*
 * PD3: fixed-length discords of length m.
 * Replaces do_PD3 + node_discords_refine + find_top1_discord
 * (src/PD3.cuh:15-61, src/sets_processing.hpp:11-46) for one series.
 *   r > 0 : one attempt at threshold r; out receives up to top_k
 *           non-overlapping discords with nn > r*r, best first.
 *   r <= 0: the halving schedule: r starts at 2*sqrt(m) and halves until
 *           top_k non-overlapping discords exist (the reference's first-length
 *           loop, src/main.cu:136-156, with the top-k condition of :137).
 * series: host pointer to n float32 values.  top_k in [1, 16].
 * segment_len: phase-1 rows per segment, 0 (the context's) or 64..4096;
 *   other values return PADDI_ERR_UNSUPPORTED.  Results do not depend on it.
 * log (optional) receives one row per attempt, at most log_cap rows.
 */
paddi_status paddi_pd3(paddi_ctx *ctx, const float *series, size_t n, uint32_t m,
                       uint32_t segment_len, uint32_t top_k, float r, paddi_discord *out,
                       uint32_t *n_out, paddi_attempt_log *log, uint32_t log_cap,
                       uint32_t *n_log);

/*
 * PALMAD: top-1 discord of every length minL..maxL with the MERLIN r-schedule
 * (src/main.cu:136-233).  out has maxL-minL+1 entries, out[k] for length minL+k.
 * series: host pointer (paddi_palmad) or device pointer (paddi_palmad_device).
 */
paddi_status paddi_palmad(paddi_ctx *ctx, const float *series, size_t n, uint32_t minL,
                          uint32_t maxL, paddi_discord *out, paddi_attempt_log *log,
                          uint32_t log_cap, uint32_t *n_log);
paddi_status paddi_palmad_device(paddi_ctx *ctx, const float *d_series, size_t n, uint32_t minL,
                                 uint32_t maxL, paddi_discord *out, paddi_attempt_log *log,
                                 uint32_t log_cap, uint32_t *n_log);

/*
 * Range-discord profile of one length, handed to a paddi_palmad_profiled
 * callback after the length's final attempt: nn[i] (N = n - m + 1 entries) is
 * the squared nn distance of window i when it is a candidate of that attempt
 * (nn >= r^2; FP64-exact near the threshold and the top, the refine's
 * estimate elsewhere) and -FLT_MAX otherwise, the nnDist layout of
 * paddi_do_pd3.  The array is valid during the call only.
 */
typedef void (*paddi_profile_fn)(void *user, uint32_t m, const float *nn, size_t N);

/*
 * paddi_palmad plus the range-discord profile of every length, passed to fn
 * in order of length.  The reference's writer for these rows is
 * write_range_discord_profile (src/IOdata.hpp:90-108: m, then the N values).
 */
paddi_status paddi_palmad_profiled(paddi_ctx *ctx, const float *series, size_t n, uint32_t minL,
                                   uint32_t maxL, paddi_discord *out, paddi_attempt_log *log,
                                   uint32_t log_cap, uint32_t *n_log, paddi_profile_fn fn,
                                   void *user);

/*
 * PALMAD over many series of uneven length (each at least 2*maxL values).
 * series[k] (host pointers) has lens[k] values; out receives count*(maxL-minL+1)
 * discords, out[k*(maxL-minL+1) + i] for series k and length minL+i; status
 * (optional, count entries) the per-series result.  The series are spread over
 * `streams` worker contexts (one CUDA stream and host thread each; 0 = 4) so
 * that their attempt pipelines overlap on the GPU.  Returns the first non-OK
 * per-series status, or PADDI_OK.  No reference counterpart (the reference runs
 * one series per invocation).
 */
paddi_status paddi_palmad_batched(paddi_ctx *ctx, const float *const *series,
                                  const size_t *lens, uint32_t count, uint32_t minL,
                                  uint32_t maxL, uint32_t streams, paddi_discord *out,
                                  int32_t *status, uint64_t *attempts);

/*
 * Autotuner: times PALMAD on short probe ranges of this series (three lengths at
 * the start, middle and end of minL..maxL) for every combination of the refine's
 * tile rows {by length, 64}, phase-1 segment length {256, 384, 512} and phase-1
 * chunk depth {8, 12, 16}, checks that all combinations return the same
 * discords, installs the fastest in ctx and copies the chosen options to
 * *chosen.  ms (optional, 18 entries) receives the probe time of each
 * combination, tile rows outermost, then segment, then chunks.  No reference
 * counterpart (the reference fixes SEGMENT_N and its 32x32 refine tiles at
 * compile time, src/parameters.hpp:8-10).
 */
paddi_status paddi_autotune(paddi_ctx *ctx, const float *series, size_t n, uint32_t minL,
                            uint32_t maxL, paddi_opts *chosen, float *ms);

/*
 * Window statistics of length m on the device, FP32 outputs.
 * Replaces compute_statistics (src/preprocessing.cuh:68-76): d_mean[i] and
 * d_std[i] (population) for i < N = n - m + 1, computed from FP64 prefix sums.
 * stream: a cudaStream_t, or NULL for the context's stream.
 */
paddi_status paddi_compute_statistics(paddi_ctx *ctx, const float *d_T, float *d_mean,
                                      float *d_std, size_t n, uint32_t m, void *stream);

/*
 * One PD3 attempt on device buffers, with the reference's output arrays.
 * Replaces do_PD3 (src/PD3.cuh:15-39) followed by node_discords_refine
 * (src/PD3.cuh:42-50): d_is_cand[i] = 1 iff window i is never pruned
 * (nn >= r2), d_nnDist[i] = its squared nn distance (FP32 estimate, FP64 near
 * the threshold) for candidates and -FLT_MAX otherwise.  r2 is squared.
 * d_T holds n values; d_is_cand / d_nnDist hold n - m + 1 entries.
 * Returns the candidate count in *n_cand.
 */
paddi_status paddi_do_pd3(paddi_ctx *ctx, const float *d_T, size_t n, uint32_t m, float r2,
                          int32_t *d_is_cand, float *d_nnDist, int64_t *n_cand, void *stream);

/* ------------------------------------------------------------------ learned r
 * A 12 -> 64 -> 64 -> 1 MLP (GELU) predicts y = log(d_m / d_{m-1}) for the
 * next length from the previous lengths (no counterpart in the reference, whose
 * schedule is src/main.cu:136-233).  Its parameters (PADDI_MODEL_NPARAM floats:
 * W1[64][12] b1[64] W2[64][64] b2[64] W3[64] b3) are trained by the library's
 * own kernels; inference runs a BF16 copy.  Under PADDI_R_LEARNED the first
 * attempt of a length starts just below the bound of PADDI_R_BOUND when that
 * bound exceeds MERLIN's first r, and otherwise uses
 * r^2 = d_{m-1} exp(y_hat) * margin, never below the bound; after a miss r^2
 * drops by at least 15% (30% from the second miss on; at least MERLIN's own
 * step), never below the bound. */
#define PADDI_MODEL_NFEAT 12
#define PADDI_MODEL_NPARAM 5057

/* Features for length minL + j from the top-1 discords of the previous lengths
 * (out[0..j-1]), the bound lb (0 if unknown), the flat-window fraction and the
 * number of attempts the previous length took.  Pure host code. */
paddi_status paddi_r_features(const paddi_discord *out, uint32_t j, uint32_t minL, float lb,
                              float flat_frac, uint32_t prev_attempts, float *features);
/* Install model parameters for PADDI_R_LEARNED; margin scales the predicted r^2. */
paddi_status paddi_model_set(paddi_ctx *ctx, const float *params, uint32_t count, float margin);
/* Train on n samples (X: n x 12 row-major, Y: n targets) with the pinball loss at
 * quantile tau, Adam, minibatches, `epochs` passes; params holds the initial
 * values on entry and the trained ones on return; loss[e] = mean loss of epoch e. */
paddi_status paddi_model_train(paddi_ctx *ctx, const float *X, const float *Y, uint32_t n,
                               float tau, uint32_t epochs, uint32_t batch, float lr,
                               uint64_t seed, float *params, float *loss);
/* Mean pinball loss and its gradient over the n samples (gradient check). */
paddi_status paddi_model_grad(paddi_ctx *ctx, const float *X, const float *Y, uint32_t n,
                              float tau, const float *params, float *grad, float *loss);
/* Forward pass for n samples with FP32 (bf16 = 0) or BF16 (bf16 = 1) weights. */
paddi_status paddi_model_predict(paddi_ctx *ctx, const float *X, uint32_t n,
                                 const float *params, int32_t bf16, float *Y);

/* ---------------------------------------------------------------- shards
 * One attempt (length m, threshold r2 = r*r) split over the GPUs of a job,
 * one process per GPU, every process holding the whole series.  Replaces the
 * reference's fragment split with halos (src/data_preparation.cuh:30-75), its
 * candidate exchange (src/MPI_transfers.hpp:29-84) and the minimum over GPUs
 * of the candidates' distances (src/sets_processing.hpp:152-164); the two
 * exchanges are the caller's (NCCL through torch.distributed, MPI, ...):
 *   1. paddi_shard_phase1: statistics of length m, then phase 1 on the rows
 *      [row_lo, row_hi) (their neighbours anywhere); writes the alive flags
 *      (uint8, 1 = not pruned) of all N = n - m + 1 windows to d_alive.
 *      Exchange: element-wise minimum of d_alive over the GPUs.
 *   2. paddi_shard_refine: the candidates of the combined flags against the
 *      windows [col_lo, col_hi) (col_lo a multiple of 2048; col_hi too, or N);
 *      writes per candidate its window (d_ind), its correlation maximum as an
 *      order-preserving uint32 image (d_rho: unsigned max = float max) and its
 *      pruned flag (d_pruned), *n_cand of them (at most cap).  Every GPU has the
 *      same candidate set, in an order of its own.
 *      Exchange: per window, the maximum of d_rho and of d_pruned over the GPUs.
 *   3. paddi_shard_select: classification, FP64 recheck and top-k of the
 *      merged candidates (count of them); the same result on every GPU.
 * The three steps run in this order on one context for one (m, r2); d_series
 * is a device pointer to n values.  log (optional) receives the attempt's row.
 */
paddi_status paddi_shard_phase1(paddi_ctx *ctx, const float *d_series, size_t n, uint32_t m,
                                float r2, size_t row_lo, size_t row_hi, uint8_t *d_alive);
paddi_status paddi_shard_refine(paddi_ctx *ctx, const float *d_series, size_t n, uint32_t m,
                                float r2, const uint8_t *d_alive, size_t col_lo, size_t col_hi,
                                int32_t *d_ind, uint32_t *d_rho, uint8_t *d_pruned, uint32_t cap,
                                uint32_t *n_cand);
paddi_status paddi_shard_select(paddi_ctx *ctx, const float *d_series, size_t n, uint32_t m,
                                float r2, const int32_t *d_ind, const uint32_t *d_rho,
                                const uint8_t *d_pruned, uint32_t count, uint32_t top_k,
                                paddi_discord *out, uint32_t *n_out, paddi_attempt_log *log);

/* The reference's MERLIN r-schedule (src/main.cu:136-233) as pure host
 * functions, for drivers outside the library: the first r of length minL + j
 * from the top-1 distances of the previous lengths (out[0..j-1]) with its
 * decrement *S, and the r after an attempt without a discord. */
float paddi_merlin_first_r(const paddi_discord *out, uint32_t j, uint32_t minL, float *S);
float paddi_merlin_lower(float r, uint32_t j, float S);

/* ------------------------------------------------------------------ test hooks
 * No counterpart in the reference, which exits the process on any CUDA error
 * (src/common.h:6-16).  These make a failure happen on the host, or make a
 * bounded device wait run out, so tests can check that the error reaches the
 * caller as a status and that the context stays usable afterwards.  Nothing
 * faults the GPU: the refine's waits all have a limit, after which the kernel
 * records the timeout, waits (bounded) for its own copies and MMAs, frees its
 * tensor memory and returns. */
typedef enum paddi_debug_key {
    PADDI_DEBUG_FAIL_ALLOC = 1,     /* value k > 0: the k-th next device allocation of the
                                       context fails (PADDI_ERR_OUT_OF_MEMORY); 0: off */
    PADDI_DEBUG_WAIT_CYCLES = 2,    /* limit of the refine's barrier waits in clock cycles
                                       (0: the default, about 2 s) */
    PADDI_DEBUG_WITHHOLD_STAGE = 3, /* 1: the next tensor-core refine launches never fill one
                                       pipeline stage, so a wait runs out (PADDI_ERR_CUDA) */
    PADDI_DEBUG_LAST_PASSES = 4,    /* read only: selection passes of the last attempt */
    PADDI_DEBUG_RECHECK_CAP = 5     /* capacity of the FP64 recheck queue (it grows on demand
                                       when a selection overflows it) */
} paddi_debug_key;
paddi_status paddi_debug_set(paddi_ctx *ctx, int32_t key, int64_t value);
paddi_status paddi_debug_get(paddi_ctx *ctx, int32_t key, int64_t *value);

/* Largest window count (n - m + 1) that paddi_compute_statistics_noalloc accepts. */
#define PADDI_NOALLOC_MAX_WINDOWS 131072

/*
 * Window statistics that allocate no device memory.
 * No counterpart in the reference: it exists for callers that may not let a
 * library call cudaMalloc, i.e. hosts that own all device memory through their
 * own allocator (managed-runtime / FFI embeddings, fixed per-tenant budgets)
 * and latency-critical loops where an allocation could synchronise the device.
 * Same results as paddi_compute_statistics (d_mean[i], d_std[i] for
 * i < n - m + 1), computed on the calling thread's current device and on
 * `stream` (a cudaStream_t; NULL is the default stream).  The kernels' scratch
 * lives in a fixed array of about 5 MB inside the library, held on every
 * device that loads the library until the process exits.
 *   - Limit: n - m + 1 <= PADDI_NOALLOC_MAX_WINDOWS, 3 <= m <= 1024, n >= 2m;
 *     anything else returns PADDI_ERR_INVALID_ARG and enqueues nothing.
 *   - The first call on a device looks up the scratch address; make it
 *     before any stream capture begins on that device.  Calls that are not
 *     under capture look it up again, so the entry point stays valid after
 *     cudaDeviceReset or from another context of the device.
 *   - All calls on a device share the scratch: calls whose GPU work overlaps
 *     (different streams or host threads) race; run them one after another.
 */
paddi_status paddi_compute_statistics_noalloc(const float *d_T, float *d_mean, float *d_std,
                                              size_t n, uint32_t m, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PADDI_H */
