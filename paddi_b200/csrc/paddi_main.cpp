// paddi_main.cpp -- command-line drop-in for the reference's PALMAD driver.
//
// Usage (positional arguments as in src/main.cu:28-33):
//   paddi-main <series.txt> <n> <minL> <maxL> <discords.csv> <times.csv>
//              [--policy merlin|bound|learned] [--dist auto|fp32|bf16|fp16]
//              [--model params.bin] [--device D] [--profile profile.csv]
// The series file holds one value per line (src/IOdata.hpp:63-88); the first
// n values are used.  Outputs follow src/IOdata.hpp:111-177: the discords file
// gets a header "m;top-1 discord idx;top-1 discord nnDist" and one row per
// length (squared distance), the times file the reference's 14 columns, one
// row per (length, r) attempt; both files are opened in append mode, as the
// reference does.  The columns for MPI exchanges and host allocation are 0
// (one GPU, one fragment, no per-attempt allocation).  --profile appends the
// range-discord profile of every length, one row "m;v_0;...;v_{N-1}" as
// src/IOdata.hpp:90-108 writes it (v_i: the window's squared nn distance when
// it is a candidate of the length's final attempt, -FLT_MAX otherwise).
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/paddi.h"

static int usage()
{
    std::fprintf(stderr,
                 "usage: paddi-main <series.txt> <n> <minL> <maxL> <discords.csv> <times.csv>\n"
                 "       [--policy merlin|bound|learned] [--dist auto|fp32|bf16|fp16]\n"
                 "       [--model params.bin] [--device D] [--profile profile.csv]\n");
    return 2;
}

int main(int argc, char **argv)
{
    if (argc < 7) return usage();
    const char *file = argv[1];
    const long long n_req = std::atoll(argv[2]);
    const int minL = std::atoi(argv[3]), maxL = std::atoi(argv[4]);
    const char *disc_file = argv[5], *times_file = argv[6];
    paddi_opts o;
    paddi_opts_default(&o);
    o.r_policy = PADDI_R_MERLIN;
    std::string model, profile;
    for (int a = 7; a + 1 < argc; a += 2) {
        const std::string k = argv[a], v = argv[a + 1];
        if (k == "--policy")
            o.r_policy = v == "bound" ? PADDI_R_BOUND : v == "learned" ? PADDI_R_LEARNED : PADDI_R_MERLIN;
        else if (k == "--dist")
            o.distance_kernel = v == "fp32" ? PADDI_DIST_FP32 : v == "bf16" ? PADDI_DIST_SPLIT_BF16
                                : v == "fp16" ? PADDI_DIST_SPLIT_FP16 : PADDI_DIST_AUTO;
        else if (k == "--model") model = v;
        else if (k == "--device") o.device = std::atoi(v.c_str());
        else if (k == "--profile") profile = v;
        else return usage();
    }
    // series: one value per line (whitespace separated), first n values
    std::vector<float> x;
    {
        std::ifstream in(file);
        if (!in) {
            std::fprintf(stderr, "cannot open %s\n", file);
            return 1;
        }
        float v;
        while ((long long)x.size() < n_req && (in >> v)) x.push_back(v);
    }
    if ((long long)x.size() < n_req)
        std::fprintf(stderr, "warning: %s holds %zu values, fewer than n = %lld\n", file, x.size(),
                     n_req);
    paddi_ctx *ctx = nullptr;
    paddi_status s = paddi_ctx_create(&ctx, &o);
    if (s != PADDI_OK) {
        std::fprintf(stderr, "paddi_ctx_create: %s\n", paddi_status_string(s));
        return 1;
    }
    if (o.r_policy == PADDI_R_LEARNED) {
        if (model.empty()) {
            std::fprintf(stderr, "--policy learned needs --model <params.bin> (%d float32)\n",
                         PADDI_MODEL_NPARAM);
            return 2;
        }
        std::vector<float> p(PADDI_MODEL_NPARAM);
        FILE *f = std::fopen(model.c_str(), "rb");
        const size_t got = f ? std::fread(p.data(), sizeof(float), p.size(), f) : 0;
        if (f) std::fclose(f);
        if (got != p.size() ||
            paddi_model_set(ctx, p.data(), PADDI_MODEL_NPARAM, 1.f) != PADDI_OK) {
            std::fprintf(stderr, "cannot load model %s\n", model.c_str());
            return 1;
        }
    }
    const int L = maxL - minL + 1;
    std::vector<paddi_discord> top(L > 0 ? L : 1);
    std::vector<paddi_attempt_log> log(1 << 16);
    uint32_t n_log = 0;
    if (profile.empty()) {
        s = paddi_palmad(ctx, x.data(), x.size(), (uint32_t)minL, (uint32_t)maxL, top.data(),
                         log.data(), (uint32_t)log.size(), &n_log);
    } else {
        std::ofstream pf(profile, std::ios::app);
        auto write_row = [](void *user, uint32_t m, const float *nn, size_t N) {
            std::ofstream &f = *static_cast<std::ofstream *>(user);
            f << m << ";";
            for (size_t i = 0; i < N; ++i) f << nn[i] << (i + 1 < N ? ";" : "\n");
        };
        s = paddi_palmad_profiled(ctx, x.data(), x.size(), (uint32_t)minL, (uint32_t)maxL,
                                  top.data(), log.data(), (uint32_t)log.size(), &n_log, write_row,
                                  &pf);
    }
    if (s != PADDI_OK) {
        std::fprintf(stderr, "paddi_palmad: %s: %s\n", paddi_status_string(s),
                     paddi_last_error(ctx));
        paddi_ctx_destroy(ctx);
        return 1;
    }
    for (int i = 0; i < L; ++i) // the reference prints each length's result
        std::printf("%d;Top-1 discord index = %d\nTop-1 discord distance = %.2f\n", minL + i,
                    top[i].ind, top[i].dist);
    {
        std::ofstream out(disc_file, std::ios::app);
        out << "m;top-1 discord idx;top-1 discord nnDist\n";
        for (int i = 0; i < L; ++i) out << minL + i << ";" << top[i].ind << ";" << top[i].dist << "\n";
    }
    {
        std::ofstream out(times_file, std::ios::app);
        out << "m;Phase1: find of segment's discords (rank = 0), ms;"
               "max statistics among GPUs (kernel), ms;max PD3 among GPUs (kernel), ms;"
               "Phase2: find of fragment's discords (rank = 0), ms;"
               "max MatrixMultiply among GPUs (kernel), ms;# Candidates;malloc memory, ms;"
               "MPI exchange C, ms;Phase3: find of global discords (rank = 0), ms;"
               "max MatrixMultiply among GPUs (kernel), ms;MPI exchange D, ms;# Discords;"
               "Total time PALMAD (rank = 0), ms\n";
        for (uint32_t i = 0; i < n_log && i < log.size(); ++i) {
            const paddi_attempt_log &e = log[i];
            out << e.m << ";" << (e.ms_stats + e.ms_phase1) << ";" << e.ms_stats << ";"
                << e.ms_phase1 << ";" << e.ms_refine << ";" << e.ms_refine << ";" << e.n_cand
                << ";0;0;" << e.ms_select << ";0;0;" << e.n_disc << ";" << e.ms_total << "\n";
        }
    }
    paddi_ctx_destroy(ctx);
    return 0;
}
