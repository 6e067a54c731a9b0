// paddi_api.cu -- host side of libpaddi: contexts, the per-attempt pipeline,
// the PD3 and PALMAD drivers and the exported C ABI (include/paddi.h).
//
// One attempt (one length m, one threshold r) is
//   phase 1     k_phase1          (reference: gpu_local_candidate_select +
//                                  gpu_local_define_candidates, src/PD3.cuh:18-29)
//   compaction  k_compact         (get_node_candidates_num + local_candidates_union,
//                                  src/sets_processing.hpp:49-113)
//   refine      k_refine_*        (gpu_local_discords_refine + gpu_global_discords_refine,
//                                  src/PD3.cuh:31-50)
//   selection   k_finalize, k_recheck, k_select
//                                 (get_node_discords_num + find_top1_discord,
//                                  src/sets_processing.hpp:11-87)
// all on one stream with one device->host copy of a small result record at
// the end.  The r-schedules are restated from src/main.cu:136-233 in the
// same float arithmetic as the reference, so equal distances give equal
// thresholds.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/paddi.h"
#include "paddi_internal.cuh"

#define PADDI_API extern "C" __attribute__((visibility("default")))

struct paddi_ctx {
    paddi_opts opts;
    int device = 0;
    int num_sms = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[6] = {};
    std::string err;
    size_t cap_n = 0; // series capacity (values)
    // device buffers
    float *d_x = nullptr;
    float4 *d_wst = nullptr;
    float *d_mu = nullptr;
    double *d_mu64 = nullptr, *d_inv64 = nullptr;
    uint8_t *d_flat = nullptr, *d_alive = nullptr, *d_pruned = nullptr;
    int32_t *d_cand = nullptr, *d_rcslot = nullptr, *d_recheck = nullptr;
    int32_t *d_list[2] = {nullptr, nullptr};
    uint32_t *d_rho = nullptr;
    unsigned long long *d_nn64 = nullptr;
    PaddiAttemptDev *d_att = nullptr;
    PaddiAttemptResult *d_res = nullptr;
    int32_t *d_flatcount = nullptr;
    PaddiAttemptResult *h_res = nullptr;
    bool umma_ok = false;
};

namespace {

const char *kStatusText[] = {"ok",
                             "invalid argument",
                             "CUDA error",
                             "out of device memory",
                             "r-schedule did not converge within the attempt cap",
                             "no sm_100 CUDA device",
                             "internal capacity exceeded",
                             "unsupported option"};

paddi_status fail(paddi_ctx *c, paddi_status s, const std::string &msg)
{
    if (c) c->err = msg;
    return s;
}

#define CK(call)                                                                            \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? PADDI_ERR_OUT_OF_MEMORY      \
                                                             : PADDI_ERR_CUDA,              \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)

template <typename T>
void dfree(T *&p)
{
    if (p) cudaFree((void *)p);
    p = nullptr;
}

void free_buffers(paddi_ctx *ctx)
{
    dfree(ctx->d_x);
    dfree(ctx->d_wst);
    dfree(ctx->d_mu);
    dfree(ctx->d_mu64);
    dfree(ctx->d_inv64);
    dfree(ctx->d_flat);
    dfree(ctx->d_alive);
    dfree(ctx->d_pruned);
    dfree(ctx->d_cand);
    dfree(ctx->d_rcslot);
    dfree(ctx->d_recheck);
    dfree(ctx->d_rho);
    dfree(ctx->d_nn64);
    dfree(ctx->d_list[0]);
    dfree(ctx->d_list[1]);
    ctx->cap_n = 0;
}

paddi_status ensure_capacity(paddi_ctx *ctx, size_t n)
{
    if (n <= ctx->cap_n) return PADDI_OK;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    free_buffers(ctx);
    const size_t W = n + PADDI_PAD_WIN + 64; // windows (upper bound) incl. the zeroed tail
    CK(cudaMalloc(&ctx->d_x, sizeof(float) * (n + 64)));
    CK(cudaMalloc(&ctx->d_wst, sizeof(float4) * W));
    CK(cudaMalloc(&ctx->d_mu, sizeof(float) * W));
    CK(cudaMalloc(&ctx->d_mu64, sizeof(double) * W));
    CK(cudaMalloc(&ctx->d_inv64, sizeof(double) * W));
    CK(cudaMalloc(&ctx->d_flat, W));
    CK(cudaMalloc(&ctx->d_alive, W));
    CK(cudaMalloc(&ctx->d_pruned, W));
    CK(cudaMalloc(&ctx->d_cand, sizeof(int32_t) * W));
    CK(cudaMalloc(&ctx->d_rcslot, sizeof(int32_t) * W));
    CK(cudaMalloc(&ctx->d_rho, sizeof(uint32_t) * W));
    CK(cudaMalloc(&ctx->d_list[0], sizeof(int32_t) * W));
    CK(cudaMalloc(&ctx->d_list[1], sizeof(int32_t) * W));
    CK(cudaMalloc(&ctx->d_recheck, sizeof(int32_t) * PADDI_MAX_RECHECK));
    CK(cudaMalloc(&ctx->d_nn64, sizeof(unsigned long long) * PADDI_MAX_RECHECK));
    CK(cudaMemsetAsync(ctx->d_wst, 0, sizeof(float4) * W, ctx->st));
    CK(cudaMemsetAsync(ctx->d_mu, 0, sizeof(float) * W, ctx->st));
    ctx->cap_n = n;
    return PADDI_OK;
}

struct AttemptOut {
    PaddiAttemptResult res;
    float ms_phase1 = 0, ms_refine = 0, ms_select = 0, ms_total = 0;
    int launches = 0;
    int kernel = PADDI_DIST_FP32;
};

// Refine kernel for length m: the tensor-core split where the length fits
// its shared-memory budget, else FP32 CUDA cores.
int refine_kernel_for(const paddi_ctx *ctx, int m)
{
    const int k = ctx->opts.distance_kernel;
    if (k == PADDI_DIST_FP32 || !ctx->umma_ok || m > paddi_umma_max_m()) return PADDI_DIST_FP32;
    return k == PADDI_DIST_SPLIT_BF16 ? PADDI_DIST_SPLIT_BF16 : PADDI_DIST_SPLIT_FP16;
}

// Correlation guard band of the pruning decisions.  FP32 and split-FP16
// keep rho within ~1e-5; split-BF16 within ~2e-4 on random-walk slices.
float guard_of(const paddi_ctx *ctx, int kernel)
{
    if (ctx->opts.guard > 0.f) return ctx->opts.guard;
    return kernel == PADDI_DIST_SPLIT_BF16 ? 1e-3f : 1e-4f;
}

// Statistics of length m for the series in `x` (n values).
paddi_status run_stats(paddi_ctx *ctx, const float *x, size_t n, int m)
{
    CK(cudaMemsetAsync(ctx->d_flatcount, 0, sizeof(int32_t), ctx->st));
    CK(paddi_launch_stats(x, (int64_t)n, m, ctx->d_wst, ctx->d_mu, ctx->d_mu64, ctx->d_inv64,
                          ctx->d_flat, ctx->d_flatcount, ctx->st));
    return PADDI_OK;
}

// One (m, r2) attempt on the statistics currently in the context.
paddi_status run_attempt(paddi_ctx *ctx, const float *x, size_t n, int m, float r2, int top_k,
                         AttemptOut *out)
{
    const int32_t N = (int32_t)(n - m + 1);
    const int kernel = refine_kernel_for(ctx, m);
    const float guard = guard_of(ctx, kernel);
    const float thr = (float)(1.0 - (double)r2 / (2.0 * (double)m));
    const float thr_prune = thr + guard;
    int R = (int)ctx->opts.segment_len;
    if (R <= 0) R = 512;
    R = (R + 7) & ~7;
    if (R < 64) R = 64;
    if (R > 1024) R = 1024;
    const int chunks = ctx->opts.phase1_chunks ? (int)ctx->opts.phase1_chunks : 4;
    cudaStream_t st = ctx->st;
    CK(cudaEventRecord(ctx->ev[0], st));
    CK(cudaMemsetAsync(ctx->d_alive, 1, (size_t)N, st));
    CK(cudaMemsetAsync(ctx->d_att, 0, sizeof(PaddiAttemptDev), st));
    int launches = 0;
    CK(paddi_launch_phase1_dev(x, ctx->d_wst, ctx->d_mu, ctx->d_alive, N, m, R, chunks, thr_prune,
                               ctx->d_flatcount, &ctx->d_att->task_next, ctx->num_sms, st));
    ++launches;
    CK(cudaEventRecord(ctx->ev[1], st));
    CK(paddi_launch_compact(ctx->d_alive, N, ctx->d_cand, ctx->d_rho, ctx->d_pruned,
                            ctx->d_rcslot, ctx->d_att, st));
    ++launches;
    // refine rounds over geometrically growing window ranges; survivors are
    // re-compacted between rounds so every tile is dense with live candidates
    CK(paddi_launch_list_init(ctx->d_att, ctx->d_list[0], &ctx->d_att->list_count[0], st));
    ++launches;
    const bool umma = kernel != PADDI_DIST_FP32;
    out->kernel = kernel;
    const int nrounds = N >= (1 << 16) ? 8 : 1;
    int jb = 0;
    for (int rd = 0; rd < nrounds; ++rd) {
        // range sizes N/128, N/128, N/64, ..., N/2 (the last round takes the rest)
        int je = rd == nrounds - 1 ? N : jb + (int)((int64_t)N >> (nrounds - (rd == 0 ? 1 : rd)));
        if (je > N) je = N;
        const int a = rd & 1, b = a ^ 1;
        CK(cudaMemsetAsync(&ctx->d_att->work_next, 0, sizeof(int32_t), st));
        if (umma)
            CK(paddi_launch_refine_umma(kernel == PADDI_DIST_SPLIT_BF16, x, ctx->d_wst, ctx->d_mu,
                                        ctx->d_cand, ctx->d_list[a],
                                        &ctx->d_att->list_count[a], ctx->d_att, ctx->d_rho,
                                        ctx->d_pruned, N, m, jb, je, thr_prune, ctx->num_sms,
                                        st));
        else
            CK(paddi_launch_refine_fp32(x, ctx->d_wst, ctx->d_mu, ctx->d_cand, ctx->d_list[a],
                                        &ctx->d_att->list_count[a], ctx->d_att, ctx->d_rho,
                                        ctx->d_pruned, N, m, jb, je, thr_prune, ctx->num_sms,
                                        st));
        ++launches;
        if (rd + 1 < nrounds) {
            CK(paddi_launch_list_compact(ctx->d_list[a], &ctx->d_att->list_count[a],
                                         ctx->d_pruned, ctx->d_list[b],
                                         &ctx->d_att->list_count[b], st));
            ++launches;
        }
        jb = je;
    }
    CK(cudaEventRecord(ctx->ev[2], st));
    float widen = 2.f;
    for (int pass = 0; pass < 3; ++pass) {
        CK(paddi_launch_finalize(ctx->d_cand, ctx->d_att, ctx->d_rho, ctx->d_pruned, m, r2, thr,
                                 guard, widen, top_k, ctx->d_flat, ctx->d_recheck,
                                 ctx->d_rcslot, ctx->d_nn64, ctx->d_res, st));
        CK(paddi_launch_recheck(x, ctx->d_mu64, ctx->d_inv64, ctx->d_flat, N, m, ctx->d_cand,
                                ctx->d_recheck, ctx->d_att, ctx->d_nn64, ctx->num_sms,
                                /*splits=*/ctx->num_sms, st));
        CK(paddi_launch_select(ctx->d_cand, ctx->d_att, ctx->d_rho, ctx->d_pruned,
                               ctx->d_recheck, ctx->d_rcslot, ctx->d_nn64, m, r2, thr, guard,
                               top_k, ctx->d_flat, ctx->d_res, st));
        launches += 3;
        CK(cudaEventRecord(ctx->ev[3], st));
        CK(cudaMemcpyAsync(ctx->h_res, ctx->d_res, sizeof(PaddiAttemptResult),
                           cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (ctx->h_res->status != 2) break;
        // a pick had no exact value: queue everything up to the cut and redo
        widen = 1e30f;
        CK(cudaMemsetAsync(&ctx->d_att->recheck_next, 0, sizeof(int32_t), st));
        CK(cudaMemsetAsync(&ctx->d_att->status, 0, sizeof(int32_t), st));
    }
    if (ctx->h_res->status == 3)
        return fail(ctx, PADDI_ERR_CUDA, "tensor-core refine: a barrier wait timed out");
    if (ctx->h_res->status == 1)
        return fail(ctx, PADDI_ERR_INTERNAL_LIMIT,
                    "more windows than the FP64 recheck capacity fall inside the guard band");
    if (ctx->h_res->status != 0)
        return fail(ctx, PADDI_ERR_INTERNAL_LIMIT, "top-k selection did not settle");
    out->res = *ctx->h_res;
    out->launches = launches;
    CK(cudaEventElapsedTime(&out->ms_phase1, ctx->ev[0], ctx->ev[1]));
    CK(cudaEventElapsedTime(&out->ms_refine, ctx->ev[1], ctx->ev[2]));
    CK(cudaEventElapsedTime(&out->ms_select, ctx->ev[2], ctx->ev[3]));
    CK(cudaEventElapsedTime(&out->ms_total, ctx->ev[0], ctx->ev[3]));
    return PADDI_OK;
}

void fill_log(paddi_attempt_log *L, int m, float r, float r2, int top_k, const AttemptOut &a,
              float ms_stats)
{
    std::memset(L, 0, sizeof(*L));
    L->m = m;
    L->r = r;
    L->r2 = r2;
    L->n_cand = a.res.n_cand;
    L->n_disc = a.res.n_disc;
    L->n_phase1 = a.res.n_p1;
    L->n_recheck = a.res.n_recheck;
    L->found = a.res.n_sel >= top_k && a.res.n_sel > 0;
    if (a.res.n_sel > 0) {
        L->top.ind = a.res.sel_ind[0];
        L->top.dist = a.res.sel_dist[0];
    } else {
        L->top.ind = -1;
        L->top.dist = -FLT_MAX;
    }
    L->ms_stats = ms_stats;
    L->ms_phase1 = a.ms_phase1;
    L->ms_refine = a.ms_refine;
    L->ms_select = a.ms_select;
    L->ms_total = a.ms_total + ms_stats;
    L->refine_pairs = (int64_t)a.res.n_pairs;
    L->n_launches = a.launches + (ms_stats > 0.f ? 1 : 0);
    L->refine_kernel = a.kernel;
}

bool valid_lengths(size_t n, uint32_t minL, uint32_t maxL)
{
    return minL >= 3 && maxL >= minL && maxL <= 1024 && n >= 2 * (size_t)maxL &&
           n < (size_t)INT32_MAX - PADDI_PAD_WIN - 64;
}

// PALMAD on a series already on the device.
paddi_status palmad_impl(paddi_ctx *ctx, const float *x, size_t n, uint32_t minL, uint32_t maxL,
                         paddi_discord *out, paddi_attempt_log *log, uint32_t log_cap,
                         uint32_t *n_log)
{
    const int L = (int)(maxL - minL + 1);
    const int iter_cap = ctx->opts.iter_cap ? (int)ctx->opts.iter_cap : 200;
    uint32_t nl = 0;
    for (int j = 0; j < L; ++j) {
        out[j].ind = -1;
        out[j].dist = -FLT_MAX;
    }
    // src/main.cu:38 -- sqrt of an unsigned int is evaluated in double
    float r = (float)(2.0 * std::sqrt((double)minL));
    for (int j = 0; j < L; ++j) {
        const int m = (int)minL + j;
        CK(cudaEventRecord(ctx->ev[4], ctx->st));
        paddi_status s = run_stats(ctx, x, n, m);
        if (s != PADDI_OK) return s;
        CK(cudaEventRecord(ctx->ev[5], ctx->st));
        float S = 0.f;
        if (j >= 1 && j < 5) {
            r = (float)((double)std::sqrt(out[j - 1].dist) * 0.99); // :171
        } else if (j >= 5) {
            float M = 0.f;
            for (int k = j - 5; k < j; ++k) M += std::sqrt(out[k].dist); // :205-206
            M = (float)((double)M * 0.2);                               // :208
            for (int k = j - 5; k < j; ++k)
                S = (float)((double)S + std::pow((double)(std::sqrt(out[k].dist) - M), 2.0));
            S = (float)std::sqrt((double)S * 0.2); // :213
            r = M - 2 * S;                         // :214
        }
        int it = 0;
        bool first = true;
        while (out[j].dist < 0) {
            if (it++ >= iter_cap)
                return fail(ctx, PADDI_ERR_ITER_CAP,
                            "length " + std::to_string(m) + ": no discord after " +
                                std::to_string(iter_cap) + " attempts");
            const float r2 = r * r;
            AttemptOut a;
            s = run_attempt(ctx, x, n, m, r2, 1, &a);
            if (s != PADDI_OK) return s;
            float ms_stats = 0.f;
            if (first) CK(cudaEventElapsedTime(&ms_stats, ctx->ev[4], ctx->ev[5]));
            first = false;
            if (a.res.n_sel > 0) {
                out[j].ind = a.res.sel_ind[0];
                out[j].dist = a.res.sel_dist[0];
            }
            if (log && nl < log_cap) fill_log(&log[nl], m, r, r2, 1, a, ms_stats);
            ++nl;
            if (j == 0) r = (float)(0.5 * (double)r);       // :155
            else if (j < 5) r = (float)(0.99 * (double)r);  // :187
            else r = r - S;                                 // :230
        }
    }
    if (n_log) *n_log = nl;
    return PADDI_OK;
}

} // namespace

// ====================================================================== ABI
PADDI_API int32_t paddi_abi_version(void) { return PADDI_ABI_VERSION; }

PADDI_API const char *paddi_status_string(paddi_status s)
{
    const int i = (int)s;
    if (i < 0 || i >= (int)(sizeof(kStatusText) / sizeof(kStatusText[0]))) return "unknown status";
    return kStatusText[i];
}

PADDI_API void paddi_opts_default(paddi_opts *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(paddi_opts);
    o->distance_kernel = PADDI_DIST_AUTO;
    o->r_policy = PADDI_R_MERLIN;
    o->segment_len = 512;
    o->phase1_chunks = 4;
    o->iter_cap = 200;
    o->guard = 0.f;
}

PADDI_API paddi_status paddi_ctx_create(paddi_ctx **out, const paddi_opts *opts)
{
    if (!out) return PADDI_ERR_INVALID_ARG;
    *out = nullptr;
    paddi_ctx *ctx = new paddi_ctx();
    paddi_opts_default(&ctx->opts);
    if (opts) {
        if (opts->struct_size != sizeof(paddi_opts)) {
            delete ctx;
            return PADDI_ERR_INVALID_ARG;
        }
        ctx->opts = *opts;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= ctx->opts.device ||
        ctx->opts.device < 0) {
        cudaGetLastError();
        delete ctx;
        return PADDI_ERR_NO_DEVICE;
    }
    ctx->device = ctx->opts.device;
    cudaDeviceProp prop;
    if (cudaSetDevice(ctx->device) != cudaSuccess ||
        cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess || prop.major < 10) {
        cudaGetLastError();
        delete ctx;
        return PADDI_ERR_NO_DEVICE;
    }
    ctx->num_sms = prop.multiProcessorCount;
    ctx->umma_ok = paddi_umma_supported(ctx->device);
    if ((ctx->opts.distance_kernel == PADDI_DIST_SPLIT_BF16 ||
         ctx->opts.distance_kernel == PADDI_DIST_SPLIT_FP16) &&
        !ctx->umma_ok) {
        delete ctx;
        return PADDI_ERR_UNSUPPORTED;
    }
    bool ok = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) == cudaSuccess;
    for (auto &e : ctx->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
    ok = ok && cudaMalloc(&ctx->d_att, sizeof(PaddiAttemptDev)) == cudaSuccess;
    ok = ok && cudaMalloc(&ctx->d_res, sizeof(PaddiAttemptResult)) == cudaSuccess;
    ok = ok && cudaMalloc(&ctx->d_flatcount, sizeof(int32_t)) == cudaSuccess;
    ok = ok && cudaMallocHost(&ctx->h_res, sizeof(PaddiAttemptResult)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        paddi_ctx_destroy(ctx);
        return PADDI_ERR_CUDA;
    }
    *out = ctx;
    return PADDI_OK;
}

PADDI_API paddi_status paddi_ctx_destroy(paddi_ctx *ctx)
{
    if (!ctx) return PADDI_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    free_buffers(ctx);
    dfree(ctx->d_att);
    dfree(ctx->d_res);
    dfree(ctx->d_flatcount);
    if (ctx->h_res) cudaFreeHost(ctx->h_res);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
    return PADDI_OK;
}

PADDI_API const char *paddi_last_error(const paddi_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

PADDI_API void *paddi_ctx_stream(paddi_ctx *ctx) { return ctx ? (void *)ctx->st : nullptr; }

PADDI_API paddi_status paddi_ctx_reserve(paddi_ctx *ctx, size_t n, uint32_t maxL)
{
    if (!ctx || n < 2 || maxL > 1024) return PADDI_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    return ensure_capacity(ctx, n);
}

PADDI_API paddi_status paddi_palmad_device(paddi_ctx *ctx, const float *d_series, size_t n,
                                           uint32_t minL, uint32_t maxL, paddi_discord *out,
                                           paddi_attempt_log *log, uint32_t log_cap,
                                           uint32_t *n_log)
{
    if (!ctx) return PADDI_ERR_INVALID_ARG;
    if (!d_series || !out || !valid_lengths(n, minL, maxL))
        return fail(ctx, PADDI_ERR_INVALID_ARG, "invalid series, lengths or output pointer");
    if (n_log) *n_log = 0;
    CK(cudaSetDevice(ctx->device));
    paddi_status s = ensure_capacity(ctx, n);
    if (s != PADDI_OK) return s;
    return palmad_impl(ctx, d_series, n, minL, maxL, out, log, log_cap, n_log);
}

PADDI_API paddi_status paddi_palmad(paddi_ctx *ctx, const float *series, size_t n, uint32_t minL,
                                    uint32_t maxL, paddi_discord *out, paddi_attempt_log *log,
                                    uint32_t log_cap, uint32_t *n_log)
{
    if (!ctx) return PADDI_ERR_INVALID_ARG;
    if (!series || !out || !valid_lengths(n, minL, maxL))
        return fail(ctx, PADDI_ERR_INVALID_ARG, "invalid series, lengths or output pointer");
    if (n_log) *n_log = 0;
    CK(cudaSetDevice(ctx->device));
    paddi_status s = ensure_capacity(ctx, n);
    if (s != PADDI_OK) return s;
    CK(cudaMemcpyAsync(ctx->d_x, series, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->st));
    return palmad_impl(ctx, ctx->d_x, n, minL, maxL, out, log, log_cap, n_log);
}

PADDI_API paddi_status paddi_pd3(paddi_ctx *ctx, const float *series, size_t n, uint32_t m,
                                 uint32_t segment_len, uint32_t top_k, float r,
                                 paddi_discord *out, uint32_t *n_out, paddi_attempt_log *log,
                                 uint32_t log_cap, uint32_t *n_log)
{
    if (!ctx) return PADDI_ERR_INVALID_ARG;
    if (!series || !out || !n_out || top_k < 1 || top_k > PADDI_MAX_TOPK ||
        !valid_lengths(n, m, m))
        return fail(ctx, PADDI_ERR_INVALID_ARG, "invalid series, length, top_k or output");
    *n_out = 0;
    if (n_log) *n_log = 0;
    CK(cudaSetDevice(ctx->device));
    paddi_status s = ensure_capacity(ctx, n);
    if (s != PADDI_OK) return s;
    const uint32_t saved_seg = ctx->opts.segment_len;
    if (segment_len) ctx->opts.segment_len = segment_len;
    CK(cudaMemcpyAsync(ctx->d_x, series, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaEventRecord(ctx->ev[4], ctx->st));
    s = run_stats(ctx, ctx->d_x, n, (int)m);
    CK(cudaEventRecord(ctx->ev[5], ctx->st));
    if (s != PADDI_OK) {
        ctx->opts.segment_len = saved_seg;
        return s;
    }
    const bool halving = !(r > 0.f);
    float rr = halving ? (float)(2.0 * std::sqrt((double)m)) : r;
    const int iter_cap = ctx->opts.iter_cap ? (int)ctx->opts.iter_cap : 200;
    uint32_t nl = 0;
    AttemptOut a;
    for (int it = 0;; ++it) {
        if (it >= iter_cap) {
            ctx->opts.segment_len = saved_seg;
            return fail(ctx, PADDI_ERR_ITER_CAP, "no discords after the attempt cap");
        }
        const float r2 = rr * rr;
        s = run_attempt(ctx, ctx->d_x, n, (int)m, r2, (int)top_k, &a);
        if (s != PADDI_OK) {
            ctx->opts.segment_len = saved_seg;
            return s;
        }
        float ms_stats = 0.f;
        if (it == 0) CK(cudaEventElapsedTime(&ms_stats, ctx->ev[4], ctx->ev[5]));
        if (log && nl < log_cap) fill_log(&log[nl], (int)m, rr, r2, (int)top_k, a, ms_stats);
        ++nl;
        const bool found = a.res.n_sel >= (int)top_k;
        if (!halving || found || r2 == 0.f) break; // r2 == 0 admits every nn > 0
        rr = (float)(0.5 * (double)rr);
    }
    ctx->opts.segment_len = saved_seg;
    *n_out = (uint32_t)a.res.n_sel;
    for (int q = 0; q < a.res.n_sel; ++q) {
        out[q].ind = a.res.sel_ind[q];
        out[q].dist = a.res.sel_dist[q];
    }
    if (n_log) *n_log = nl;
    return PADDI_OK;
}

PADDI_API paddi_status paddi_compute_statistics(paddi_ctx *ctx, const float *d_T, float *d_mean,
                                                float *d_std, size_t n, uint32_t m, void *stream)
{
    if (!ctx) return PADDI_ERR_INVALID_ARG;
    if (!d_T || !d_mean || !d_std || !valid_lengths(n, m, m))
        return fail(ctx, PADDI_ERR_INVALID_ARG, "invalid pointers or length");
    CK(cudaSetDevice(ctx->device));
    paddi_status s = ensure_capacity(ctx, n);
    if (s != PADDI_OK) return s;
    cudaStream_t user = stream ? (cudaStream_t)stream : ctx->st;
    if (user != ctx->st) { // order the context stream after the caller's
        CK(cudaEventRecord(ctx->ev[4], user));
        CK(cudaStreamWaitEvent(ctx->st, ctx->ev[4], 0));
    }
    s = run_stats(ctx, d_T, n, (int)m);
    if (s != PADDI_OK) return s;
    CK(paddi_launch_export_stats(ctx->d_mu64, ctx->d_inv64, (int32_t)(n - m + 1), (int)m, d_mean,
                                 d_std, ctx->st));
    if (user != ctx->st) {
        CK(cudaEventRecord(ctx->ev[5], ctx->st));
        CK(cudaStreamWaitEvent(user, ctx->ev[5], 0));
    }
    return PADDI_OK;
}

PADDI_API paddi_status paddi_do_pd3(paddi_ctx *ctx, const float *d_T, size_t n, uint32_t m,
                                    float r2, int32_t *d_is_cand, float *d_nnDist,
                                    int64_t *n_cand, void *stream)
{
    if (!ctx) return PADDI_ERR_INVALID_ARG;
    if (!d_T || !d_is_cand || !d_nnDist || !valid_lengths(n, m, m) || !(r2 >= 0.f))
        return fail(ctx, PADDI_ERR_INVALID_ARG, "invalid pointers, length or threshold");
    CK(cudaSetDevice(ctx->device));
    paddi_status s = ensure_capacity(ctx, n);
    if (s != PADDI_OK) return s;
    cudaStream_t user = stream ? (cudaStream_t)stream : ctx->st;
    if (user != ctx->st) {
        CK(cudaEventRecord(ctx->ev[4], user));
        CK(cudaStreamWaitEvent(ctx->st, ctx->ev[4], 0));
    }
    s = run_stats(ctx, d_T, n, (int)m);
    if (s != PADDI_OK) return s;
    AttemptOut a;
    s = run_attempt(ctx, d_T, n, (int)m, r2, 1, &a);
    if (s != PADDI_OK) return s;
    CK(paddi_launch_scatter(ctx->d_cand, ctx->d_att, ctx->d_rho, ctx->d_pruned, ctx->d_rcslot,
                            ctx->d_nn64, ctx->d_flat, (int32_t)(n - m + 1), (int)m, r2, d_is_cand,
                            d_nnDist, ctx->st));
    if (user != ctx->st) {
        CK(cudaEventRecord(ctx->ev[5], ctx->st));
        CK(cudaStreamWaitEvent(user, ctx->ev[5], 0));
    } else {
        CK(cudaStreamSynchronize(ctx->st));
    }
    if (n_cand) *n_cand = a.res.n_cand;
    return PADDI_OK;
}
