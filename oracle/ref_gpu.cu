// ref_gpu.cu -- C-linkage driver around the reference's own FP32 GPU kernels.
//
// TEST / BASELINE INFRASTRUCTURE ONLY.  The product library never links or
// loads it.  oracle/Makefile compiles it with nvcc against the reference's
// headers where they lie (src/PD3_kernels.cuh, src/preprocessing.cuh,
// src/parameters.hpp, unmodified) into oracle/_ref/libpaddi_refgpu.so; bench.py
// times it as the "reference FP32 GPU" point beside the library.
//
// The reference's per-length driver (do_PALMAD_one_length) is not in its
// source tree (src/main.cu:20 includes a missing PALMAD_one_length.cuh), so
// one attempt is restated from the pieces that exist, for one GPU and one
// fragment:
//   compute_statistics                      src/preprocessing.cuh:68-76
//   do_PD3: phase 1, define, local refine   src/PD3.cuh:15-39 (same launch
//                                           shapes; its per-call printf left out)
//   local_candidates_union (host gather)    src/sets_processing.hpp:90-113
//   node_discords_refine                    src/PD3.cuh:42-50
//   find_top1_discord                       src/sets_processing.hpp:11-46
// with the series padded as the reference pads it (FLT_MAX values up to a
// multiple of SEGMENT_N plus an (m - 1) halo, src/data_preparation.cuh:12-28,
// src/IOdata.hpp) and every device array given 4096 more padded entries, so
// no launch shape can read past an allocation.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "PD3_kernels.cuh"
#include "preprocessing.cuh"

namespace {

constexpr size_t kSlack = 4096;

struct RefAttempt {
    int32_t m;
    float r2;
    int64_t n_cand;   // candidates after phase 1, define and the local refine
    int64_t n_disc;   // candidates with nnDist > r2 after the node refine
    int32_t top_ind;
    float top_dist;
    float ms;         // device time of the attempt (statistics to top-1)
};

template <typename T>
struct Dev {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count)
    {
        if (count <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, sizeof(T) * count);
        if (e == cudaSuccess) n = count;
        return e;
    }
    ~Dev()
    {
        if (p) cudaFree(p);
    }
};

#define RCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return (int)e_;                                                     \
    } while (0)

} // namespace

extern "C" {

// One attempt of the reference's FP32 GPU path at length m and squared
// threshold r2 on the host series x (n values).  Returns 0 or a cudaError_t.
__attribute__((visibility("default"))) int refgpu_attempt(const float *x, int64_t n, int32_t m,
                                                          float r2, RefAttempt *out)
{
    const unsigned N_real = (unsigned)(n - m + 1);
    if ((N_real + BLOCK_DIM - 1) / BLOCK_DIM > 65535u) // the node refine's 2-D grid
        return (int)cudaErrorInvalidConfiguration;
    const unsigned k = (N_real + SEGMENT_N - 1) / SEGMENT_N;
    const unsigned N_pad = k * SEGMENT_N + m - 1;   // windows incl. padding
    const unsigned n_pad = N_pad + m - 1;           // values incl. padding
    std::vector<float> h((size_t)n_pad + kSlack, FLT_MAX);
    std::memcpy(h.data(), x, sizeof(float) * (size_t)n);
    Dev<float> T, mu, sd, nn, Cm, cnn;
    Dev<int> isc, isn, cidx;
    RCK(T.alloc(h.size()));
    RCK(mu.alloc((size_t)N_pad + kSlack));
    RCK(sd.alloc((size_t)N_pad + kSlack));
    RCK(nn.alloc((size_t)N_pad + kSlack));
    RCK(isc.alloc((size_t)N_pad + kSlack));
    RCK(isn.alloc((size_t)N_pad + kSlack));
    cudaStream_t st;
    RCK(cudaStreamCreate(&st));
    cudaEvent_t e0, e1;
    RCK(cudaEventCreate(&e0));
    RCK(cudaEventCreate(&e1));
    RCK(cudaMemcpyAsync(T.p, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, st));
    std::vector<int> ones((size_t)N_pad + kSlack, 1);
    std::vector<float> fmax((size_t)N_pad + kSlack, FLT_MAX);
    RCK(cudaMemcpyAsync(isc.p, ones.data(), sizeof(int) * ones.size(), cudaMemcpyHostToDevice, st));
    RCK(cudaMemcpyAsync(isn.p, ones.data(), sizeof(int) * ones.size(), cudaMemcpyHostToDevice, st));
    RCK(cudaMemcpyAsync(nn.p, fmax.data(), sizeof(float) * fmax.size(), cudaMemcpyHostToDevice,
                        st));
    RCK(cudaMemsetAsync(mu.p, 0, sizeof(float) * mu.n, st));
    RCK(cudaMemsetAsync(sd.p, 0, sizeof(float) * sd.n, st));
    RCK(cudaEventRecord(e0, st));
    // statistics of all padded windows (src/preprocessing.cuh:68-76)
    compute_statistics(T.p, mu.p, sd.p, N_pad, (unsigned)m, st);
    // do_PD3 (src/PD3.cuh:15-39): N = the padded series length
    const unsigned Nser = n_pad;
    {
        unsigned nb = (Nser - m + 1) / SEGMENT_N;
        gpu_local_candidate_select<<<nb, SEGMENT_N, (2 * SEGMENT_N + 2 * m - 2) * sizeof(float),
                                     st>>>(T.p, mu.p, sd.p, isc.p, isn.p, nn.p, Nser, (int)N_real,
                                           r2, (unsigned)m, 0);
        nb = (unsigned)std::ceil(Nser / (float)DEFINE_CAND_BLOCK_SIZE);
        gpu_local_define_candidates<<<nb, DEFINE_CAND_BLOCK_SIZE, 0, st>>>(isc.p, isn.p, Nser, 0);
        nb = (Nser - m + 1) / SEGMENT_N;
        gpu_local_discords_refine<<<nb, SEGMENT_N, (2 * SEGMENT_N + 2 * m - 2) * sizeof(float),
                                    st>>>(T.p, mu.p, sd.p, isc.p, nn.p, Nser, (unsigned)m, r2);
    }
    RCK(cudaGetLastError());
    // candidates to the host and the union (src/sets_processing.hpp:90-113)
    std::vector<int> hc(N_real);
    RCK(cudaMemcpyAsync(hc.data(), isc.p, sizeof(int) * N_real, cudaMemcpyDeviceToHost, st));
    RCK(cudaStreamSynchronize(st));
    std::vector<int> idx;
    for (unsigned i = 0; i < N_real; ++i)
        if (hc[i]) idx.push_back((int)i);
    const unsigned C = (unsigned)idx.size();
    out->m = m;
    out->r2 = r2;
    out->n_cand = C;
    out->n_disc = 0;
    out->top_ind = -1;
    out->top_dist = -FLT_MAX;
    if (C > 0) {
        const size_t Cp = ((size_t)C + 31) / 32 * 32 + kSlack;
        std::vector<float> hC((size_t)m * C);
        for (unsigned c = 0; c < C; ++c)
            for (int q = 0; q < m; ++q) hC[(size_t)C * q + c] = h[(size_t)idx[c] + q];
        std::vector<int> hidx(Cp, 0);
        std::memcpy(hidx.data(), idx.data(), sizeof(int) * C);
        std::vector<float> hnn(Cp, FLT_MAX);
        RCK(Cm.alloc(hC.size() + kSlack));
        RCK(cidx.alloc(Cp));
        RCK(cnn.alloc(Cp));
        RCK(cudaMemcpyAsync(Cm.p, hC.data(), sizeof(float) * hC.size(), cudaMemcpyHostToDevice,
                            st));
        RCK(cudaMemcpyAsync(cidx.p, hidx.data(), sizeof(int) * Cp, cudaMemcpyHostToDevice, st));
        RCK(cudaMemcpyAsync(cnn.p, hnn.data(), sizeof(float) * Cp, cudaMemcpyHostToDevice, st));
        // node_discords_refine (src/PD3.cuh:42-50) over the one fragment
        dim3 bd(BLOCK_DIM, BLOCK_DIM, 1);
        dim3 gd((unsigned)std::ceil(C / (float)BLOCK_DIM), (unsigned)std::ceil(N_real / (float)BLOCK_DIM),
                1);
        gpu_global_discords_refine<<<gd, bd, 0, st>>>(T.p, mu.p, sd.p, Cm.p, cidx.p, cnn.p,
                                                       (int)N_real, (int)N_real, (int)C,
                                                       (unsigned)m, r2, 0);
        RCK(cudaGetLastError());
        std::vector<float> res(C);
        RCK(cudaMemcpyAsync(res.data(), cnn.p, sizeof(float) * C, cudaMemcpyDeviceToHost, st));
        RCK(cudaEventRecord(e1, st));
        RCK(cudaStreamSynchronize(st));
        // find_top1_discord (src/sets_processing.hpp:11-46), one process
        float best = -FLT_MAX;
        for (unsigned c = 0; c < C; ++c) {
            const float v = res[c];
            if (v > best && v > r2) {
                best = v;
                out->top_ind = idx[c];
                out->top_dist = v;
            }
            if (v > r2) ++out->n_disc;
        }
    } else {
        RCK(cudaEventRecord(e1, st));
        RCK(cudaStreamSynchronize(st));
    }
    float ms = 0.f;
    RCK(cudaEventElapsedTime(&ms, e0, e1));
    out->ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    return 0;
}

struct RefDiscord {
    int32_t ind;
    float dist;
};

// PALMAD over minL..maxL with the reference's FP32 GPU path and its MERLIN
// schedule (src/main.cu:136-233, the same float arithmetic as ref_wrap.cpp's
// CPU driver), stopping at the first length boundary after max_attempts
// attempts.  Returns the number of lengths completed (out[0..] filled), or
// -(cudaError_t) on a CUDA error; *n_att: attempts run, *ms: their device time.
__attribute__((visibility("default"))) int32_t refgpu_palmad(const float *x, int64_t n,
                                                             int32_t minL, int32_t maxL,
                                                             int32_t iter_cap, int32_t max_attempts,
                                                             RefDiscord *out, int32_t *n_att,
                                                             double *ms)
{
    const int32_t L = maxL - minL + 1;
    for (int32_t j = 0; j < L; ++j) {
        out[j].ind = -1;
        out[j].dist = -FLT_MAX;
    }
    *n_att = 0;
    *ms = 0.0;
    float r = 2 * std::sqrt(minL); // src/main.cu:38
    for (int32_t j = 0; j < L; ++j) {
        if (*n_att >= max_attempts) return j;
        const int32_t m = minL + j;
        float S = 0;
        if (j >= 1 && j < 5) {
            r = std::sqrt(out[j - 1].dist) * 0.99;
        } else if (j >= 5) {
            float M = 0;
            for (int k = j - 5; k < j; ++k) M += std::sqrt(out[k].dist);
            M = M * 0.2;
            for (int k = j - 5; k < j; ++k) S += std::pow((std::sqrt(out[k].dist) - M), 2);
            S = std::sqrt(S * 0.2);
            r = M - 2 * S;
        }
        for (int32_t it = 0; out[j].dist < 0; ++it) {
            if (it >= iter_cap) return j;
            RefAttempt a;
            const int e = refgpu_attempt(x, n, m, r * r, &a);
            if (e) return -e;
            ++*n_att;
            *ms += a.ms;
            if (a.top_ind >= 0) {
                out[j].ind = a.top_ind;
                out[j].dist = a.top_dist;
            }
            if (j == 0) r = 0.5 * r;
            else if (j < 5) r = 0.99 * r;
            else r = r - S;
        }
    }
    return L;
}

} // extern "C"
