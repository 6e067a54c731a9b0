// ref_wrap.cpp -- C-linkage driver around the reference's own CPU kernels.
//
// TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline).  It is linked
// with the reference's src/cpu_kernels/cpu_kernels.cpp, compiled unmodified
// from where it lies, into oracle/_ref/libpaddi_ref.so by oracle/Makefile.
//
// The reference's do_PALMAD_one_length is not part of its source tree
// (src/main.cu:20 includes a missing PALMAD_one_length.cuh), so the CPU path
// of one (length, r) attempt is restated here from the pieces that exist:
//   compute_statistics_cpu            src/cpu_kernels/cpu_kernels.cpp:7-31
//   find_discords_cpu                 src/cpu_kernels/cpu_kernels.cpp:33-78
//   find_top1_discord semantics       src/sets_processing.hpp:11-46
// and the MERLIN r-schedule of src/main.cu:136-233 drives it.
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <atomic>
#include <thread>
#include <vector>

#include "cpu_kernels.hpp"

extern "C" {

struct ref_discord {
    int32_t ind;
    float dist;
};

struct ref_attempt {
    int32_t m;
    float r;
    float r2;
    int64_t n_cand;
    int64_t n_disc;
    int32_t found;
    int32_t n_sel;
    ref_discord top;
};

__attribute__((visibility("default"))) void ref_compute_statistics(float *T, float *mean,
                                                                   float *sd, uint32_t N,
                                                                   uint32_t m)
{
    compute_statistics_cpu(T, mean, sd, N, m);
}

__attribute__((visibility("default"))) void ref_find_discords(float *T, float *mean, float *sd,
                                                              int32_t *cand, float *nnDist,
                                                              uint32_t N, float r2, uint32_t m)
{
    find_discords_cpu(T, mean, sd, cand, nnDist, N, r2, m);
}

// One attempt: statistics, brute-force range discords, top-1 over the
// survivors with nnDist > r2 (strict, first maximum).
static ref_attempt one_attempt(float *T, int64_t n, int32_t m, float r, std::vector<float> &mu,
                               std::vector<float> &sd, std::vector<int32_t> &cand,
                               std::vector<float> &nnd)
{
    const uint32_t N = (uint32_t)(n - m + 1);
    compute_statistics_cpu(T, mu.data(), sd.data(), N, (uint32_t)m);
    for (uint32_t i = 0; i < N; ++i) {
        cand[i] = 1;
        nnd[i] = FLT_MAX;
    }
    const float r2 = r * r;
    find_discords_cpu(T, mu.data(), sd.data(), cand.data(), nnd.data(), N, r2, (uint32_t)m);
    ref_attempt a;
    std::memset(&a, 0, sizeof(a));
    a.m = m;
    a.r = r;
    a.r2 = r2;
    a.top.ind = -1;
    a.top.dist = -FLT_MAX;
    float best = -FLT_MAX;
    for (uint32_t i = 0; i < N; ++i) {
        if (!cand[i]) continue;
        ++a.n_cand;
        if (nnd[i] > r2) {
            ++a.n_disc;
            if (nnd[i] > best) {
                best = nnd[i];
                a.top.ind = (int32_t)i;
                a.top.dist = nnd[i];
            }
        }
    }
    a.found = a.top.ind >= 0;
    a.n_sel = a.found;
    return a;
}

// PALMAD over minL..maxL with the reference CPU kernels; returns the number
// of attempts (or -1 when a length exceeded iter_cap attempts).
__attribute__((visibility("default"))) int64_t ref_palmad(float *T, int64_t n, int32_t minL,
                                                          int32_t maxL, int32_t iter_cap,
                                                          ref_discord *out, ref_attempt *log,
                                                          int64_t log_cap)
{
    const int32_t L = maxL - minL + 1;
    std::vector<float> mu(n), sd(n), nnd(n);
    std::vector<int32_t> cand(n);
    for (int32_t j = 0; j < L; ++j) {
        out[j].ind = -1;
        out[j].dist = -FLT_MAX;
    }
    int64_t natt = 0;
    float r = 2 * std::sqrt(minL); // src/main.cu:38 (sqrt of an integer -> double)
    for (int32_t j = 0; j < L; ++j) {
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
        int32_t it = 0;
        while (out[j].dist < 0) {
            if (it++ >= iter_cap) return -1;
            ref_attempt a = one_attempt(T, n, m, r, mu, sd, cand, nnd);
            out[j] = a.top;
            if (log && natt < log_cap) log[natt] = a;
            ++natt;
            if (j == 0) r = 0.5 * r;
            else if (j < 5) r = 0.99 * r;
            else r = r - S;
        }
    }
    return natt;
}

// Fixed-length attempt at a given r (linear), for parity fixtures.
__attribute__((visibility("default"))) void ref_attempt_at(float *T, int64_t n, int32_t m,
                                                           float r, ref_attempt *att,
                                                           int32_t *cand_out, float *nn_out)
{
    const int64_t N = n - m + 1;
    std::vector<float> mu(n), sd(n), nnd(n);
    std::vector<int32_t> cand(n);
    *att = one_attempt(T, n, m, r, mu, sd, cand, nnd);
    if (cand_out) std::memcpy(cand_out, cand.data(), sizeof(int32_t) * N);
    if (nn_out) std::memcpy(nn_out, nnd.data(), sizeof(float) * N);
}

// Run independent PALMAD jobs on `threads` host threads (one series slice
// per job, handed out in order to whichever thread is free).  The reference kernels are pure functions of their arguments,
// so concurrent calls on disjoint buffers are safe.
__attribute__((visibility("default"))) int64_t ref_palmad_many(float *const *series,
                                                               const int64_t *lens, int32_t jobs,
                                                               int32_t minL, int32_t maxL,
                                                               int32_t iter_cap, int32_t threads,
                                                               ref_discord *out)
{
    const int32_t L = maxL - minL + 1;
    std::vector<int64_t> natt(jobs, 0);
    std::vector<std::thread> pool;
    std::atomic<int32_t> next{0};
    for (int32_t t = 0; t < threads; ++t) {
        pool.emplace_back([&]() {
            for (int32_t k; (k = next.fetch_add(1)) < jobs;)
                natt[k] = ref_palmad(series[k], lens[k], minL, maxL, iter_cap,
                                     out + (size_t)k * L, nullptr, 0);
        });
    }
    for (auto &th : pool) th.join();
    int64_t total = 0;
    for (int32_t k = 0; k < jobs; ++k) {
        if (natt[k] < 0) return -1;
        total += natt[k];
    }
    return total;
}

} // extern "C"
