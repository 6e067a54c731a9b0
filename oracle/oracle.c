/*
 * oracle.c -- FP64 CPU restatement of the PADDi discord-discovery path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, as the checker.
 *
 * What it restates (paths relative to the PADDi source tree):
 *   - window mean / population std         src/preprocessing.cuh:24-34
 *   - squared z-normalised distance         src/PD3_kernels.cuh:61,102,179,213
 *       d = 2m (1 - (QT - m mu_i mu_j) / (m sd_i sd_j))
 *     evaluated here in the centred, exact form d = 2m (1 - rho) with
 *     rho = sum_k (x_i+k - mu_i)(x_j+k - mu_j) / (|x_i - mu_i| |x_j - mu_j|).
 *   - trivial-match exclusion |i - j| < m-1 src/PD3_kernels.cuh:70,114,458,491
 *     (the CPU kernel's |i-1-j| < m, src/cpu_kernels/cpu_kernels.cpp:57, is
 *     available through the right_gap/left_gap parameters)
 *   - pruning: a window stops being a candidate as soon as one admissible
 *     neighbour has d < r                   src/PD3_kernels.cuh:74-78,372-376
 *   - discord test nnDist > r, top-1 = first (lowest index) maximum
 *                                           src/sets_processing.hpp:11-46
 *   - the MERLIN r-schedule across lengths  src/main.cu:136-233
 *
 * Policies where the reference's FP32 arithmetic is not well defined
 * (documented; the GPU library follows the same policies):
 *   - a window whose m values are all equal is "flat" (sd = 0).  A pair with
 *     exactly one flat window has rho = 0 (d = 2m: the reference maps the
 *     resulting x/0 = inf to 2m, src/PD3_kernels.cuh:63-64); a pair of two
 *     flat windows has rho = 1 (d = 0: the reference's 0/0 = NaN is mapped
 *     to -FLT_MAX, i.e. "closer than any r", src/PD3_kernels.cuh:107-108).
 *   - d is clamped below at 0.  Exact arithmetic never gives d < 0; the
 *     reference's "d < 0 -> 2m" clamp (src/PD3_kernels.cuh:63) only fires on
 *     FP32 rounding of near-identical windows.
 *
 * The r-schedule is restated in float32 with the same operation order and
 * the same float/double promotions as the reference (C++ overloads of sqrt
 * and pow on float), so identical distances give identical r sequences.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* window statistics                                                    */
/* ------------------------------------------------------------------ */

/* mu[i], sd[i] (population) of x[i..i+m), i < N = n-m+1; two-pass in FP64.
 * flat[i] = 1 iff all m values are equal (then sd[i] = 0 exactly). */
OR_EXPORT void or_window_stats(const float *x, int64_t n, int32_t m,
                               double *mu, double *sd, uint8_t *flat)
{
    const int64_t N = n - m + 1;
    /* run[i] = number of equal values starting at i (exact integer test) */
    int64_t run = 1;
    int64_t *runs = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    runs[n - 1] = 1;
    for (int64_t i = n - 2; i >= 0; --i) {
        run = (x[i] == x[i + 1]) ? run + 1 : 1;
        runs[i] = run;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        double s = 0.0;
        for (int32_t k = 0; k < m; ++k) s += (double)x[i + k];
        const double u = s / m;
        double v = 0.0;
        for (int32_t k = 0; k < m; ++k) {
            const double d = (double)x[i + k] - u;
            v += d * d;
        }
        const int f = runs[i] >= m;
        mu[i] = f ? (double)x[i] : u;
        sd[i] = f ? 0.0 : sqrt(v / m);
        if (flat) flat[i] = (uint8_t)f;
    }
    free(runs);
}

/* ------------------------------------------------------------------ */
/* nearest-neighbour profile                                            */
/* ------------------------------------------------------------------ */

typedef struct {
    int64_t n, N;
    int32_t m;
    const float *x;
    double *mu, *inv; /* inv = 1 / |x_i - mu_i|, 0 for flat */
    uint8_t *flat;
} or_series;

static void series_init(or_series *s, const float *x, int64_t n, int32_t m)
{
    s->n = n;
    s->m = m;
    s->N = n - m + 1;
    s->x = x;
    s->mu = (double *)malloc(sizeof(double) * (size_t)s->N);
    s->inv = (double *)malloc(sizeof(double) * (size_t)s->N);
    s->flat = (uint8_t *)malloc((size_t)s->N);
    double *sd = (double *)malloc(sizeof(double) * (size_t)s->N);
    or_window_stats(x, n, m, s->mu, sd, s->flat);
    for (int64_t i = 0; i < s->N; ++i)
        s->inv[i] = s->flat[i] ? 0.0 : 1.0 / (sd[i] * sqrt((double)m));
    free(sd);
}

static void series_free(or_series *s)
{
    free(s->mu);
    free(s->inv);
    free(s->flat);
}

/* centred covariance sum_k (x_i+k - mu_i)(x_j+k - mu_j), direct O(m) */
static double cov_direct(const or_series *s, int64_t i, int64_t j)
{
    const float *a = s->x + i, *b = s->x + j;
    const double ua = s->mu[i], ub = s->mu[j];
    double acc = 0.0;
    for (int32_t k = 0; k < s->m; ++k) acc += ((double)a[k] - ua) * ((double)b[k] - ub);
    return acc;
}

static inline double dist_from_cov(const or_series *s, int64_t i, int64_t j, double cov)
{
    double rho;
    if (s->flat[i] | s->flat[j])
        rho = (s->flat[i] & s->flat[j]) ? 1.0 : 0.0;
    else
        rho = cov * s->inv[i] * s->inv[j];
    double d = 2.0 * s->m * (1.0 - rho);
    return d < 0.0 ? 0.0 : d;
}

/* d(i, j) in FP64 (direct). */
OR_EXPORT double or_pair_dist(const float *x, int64_t n, int32_t m, int64_t i, int64_t j)
{
    or_series s;
    series_init(&s, x, n, m);
    const double d = dist_from_cov(&s, i, j, cov_direct(&s, i, j));
    series_free(&s);
    return d;
}

static inline void upd(double *nn, int64_t *idx, int64_t i, double d, int64_t j)
{
    if (d < nn[i] || (d == nn[i] && j < idx[i])) {
        nn[i] = d;
        idx[i] = j;
    }
}

/*
 * nn[i] = min over admissible j of d(i, j); idx[i] = the lowest such j.
 * j is admissible for row i iff  j - i >= right_gap  or  i - j >= left_gap
 * (GPU rule: right_gap = left_gap = m-1; CPU kernel rule: m-1 and m+1).
 * Windows without any admissible neighbour get nn = +inf, idx = -1.
 * method 0: direct O(N^2 m); method 1: FP64 diagonal recurrence O(N^2)
 * (covariance update of the published mpx/SCAMP form, re-anchored by a
 * direct dot product every 64 steps).
 */
OR_EXPORT void or_nn_profile(const float *x, int64_t n, int32_t m, int32_t right_gap,
                             int32_t left_gap, int32_t method, double *nn, int64_t *idx)
{
    or_series s;
    series_init(&s, x, n, m);
    const int64_t N = s.N;
    const int32_t gmin = right_gap < left_gap ? right_gap : left_gap;
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    double *tnn = (double *)malloc(sizeof(double) * (size_t)N * nth);
    int64_t *tix = (int64_t *)malloc(sizeof(int64_t) * (size_t)N * nth);
    for (int64_t k = 0; k < N * nth; ++k) {
        tnn[k] = INFINITY;
        tix[k] = INT64_MAX;
    }
    double *df = NULL, *dg = NULL;
    if (method == 1) {
        df = (double *)malloc(sizeof(double) * (size_t)N);
        dg = (double *)malloc(sizeof(double) * (size_t)N);
        for (int64_t i = 0; i + 1 < N; ++i) {
            df[i] = ((double)x[i + m] - (double)x[i]) * 0.5;
            dg[i] = ((double)x[i + m] - s.mu[i + 1]) + ((double)x[i] - s.mu[i]);
        }
    }
#pragma omp parallel
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double *mnn = tnn + (size_t)t * N;
        int64_t *mix = tix + (size_t)t * N;
#pragma omp for schedule(dynamic, 16)
        for (int64_t dlt = gmin > 0 ? gmin : 1; dlt < N; ++dlt) {
            const int row_ok = dlt >= right_gap; /* j = i+dlt is a right neighbour of i */
            const int col_ok = dlt >= left_gap;  /* i is a left neighbour of j */
            if (!row_ok && !col_ok) continue;
            double cov = 0.0;
            for (int64_t i = 0; i + dlt < N; ++i) {
                const int64_t j = i + dlt;
                if (method == 0 || (i & 63) == 0)
                    cov = cov_direct(&s, i, j);
                const double d = dist_from_cov(&s, i, j, cov);
                if (row_ok) upd(mnn, mix, i, d, j);
                if (col_ok) upd(mnn, mix, j, d, i);
                if (method == 1 && j + 1 < N) cov += df[i] * dg[j] + df[j] * dg[i];
            }
        }
    }
    for (int64_t i = 0; i < N; ++i) {
        double b = INFINITY;
        int64_t bj = INT64_MAX;
        for (int t = 0; t < nth; ++t) {
            const double d = tnn[(size_t)t * N + i];
            const int64_t j = tix[(size_t)t * N + i];
            if (d < b || (d == b && j < bj)) {
                b = d;
                bj = j;
            }
        }
        nn[i] = b;
        idx[i] = bj == INT64_MAX ? -1 : bj;
    }
    free(tnn);
    free(tix);
    free(df);
    free(dg);
    series_free(&s);
}

/*
 * nn[i] = min over admissible j (|i - j| >= m-1) of d(i, j), FP64, for long
 * series: the same diagonal recurrence as or_nn_profile method 1, over blocks
 * of 8 neighbouring diagonals so the inner loop vectorises, re-anchored by a
 * direct dot product every 8192 rows (the FP64 recurrence drifts by ~1e-12 of
 * n_i n_j over that many steps).  Pairs with a flat window get d = 2m in the
 * loop; flat windows are settled afterwards by the flat-window rule (d = 0 to
 * any admissible flat window).  Windows without an admissible neighbour get
 * +inf.  Only nn is returned (no index).
 */
#define PB_D 8
#define PB_ANCHOR 8192
OR_EXPORT void or_nn_profile_fast(const float *x, int64_t n, int32_t m, double *nn)
{
    or_series s;
    series_init(&s, x, n, m);
    const int64_t N = s.N;
    const int32_t gap = m - 1;
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    double *tnn = (double *)malloc(sizeof(double) * (size_t)(N + PB_D) * nth);
    for (int64_t k = 0; k < (N + PB_D) * nth; ++k) tnn[k] = INFINITY;
    double *df = (double *)calloc((size_t)(N + PB_D), sizeof(double));
    double *dg = (double *)calloc((size_t)(N + PB_D), sizeof(double));
    double *iv = (double *)calloc((size_t)(N + PB_D), sizeof(double));
    for (int64_t i = 0; i + 1 < N; ++i) {
        df[i] = ((double)x[i + m] - (double)x[i]) * 0.5;
        dg[i] = ((double)x[i + m] - s.mu[i + 1]) + ((double)x[i] - s.mu[i]);
    }
    for (int64_t i = 0; i < N; ++i) iv[i] = s.inv[i];
    const double twom = 2.0 * m;
    const int64_t nblk = N > gap ? (N - gap + PB_D - 1) / PB_D : 0;
#pragma omp parallel
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double *mnn = tnn + (size_t)t * (N + PB_D);
#pragma omp for schedule(dynamic, 4)
        for (int64_t b = 0; b < nblk; ++b) {
            const int64_t d0 = gap + b * PB_D;
            double cov[PB_D];
            /* rows i with i + d0 + PB_D - 1 < N: all 8 diagonals in range */
            const int64_t full = N - (d0 + PB_D - 1);
            for (int64_t i0 = 0; i0 < full; i0 += PB_ANCHOR) {
                const int64_t i1 = i0 + PB_ANCHOR < full ? i0 + PB_ANCHOR : full;
                for (int k = 0; k < PB_D; ++k) cov[k] = cov_direct(&s, i0, i0 + d0 + k);
                for (int64_t i = i0; i < i1; ++i) {
                    const double ivi = iv[i], dfi = df[i], dgi = dg[i];
                    const int64_t j = i + d0;
                    double rmin = mnn[i];
#pragma omp simd reduction(min : rmin)
                    for (int k = 0; k < PB_D; ++k) {
                        double d = twom * (1.0 - cov[k] * ivi * iv[j + k]);
                        d = d < 0.0 ? 0.0 : d;
                        rmin = d < rmin ? d : rmin;
                        mnn[j + k] = d < mnn[j + k] ? d : mnn[j + k];
                        cov[k] += dfi * dg[j + k] + df[j + k] * dgi;
                    }
                    mnn[i] = rmin;
                }
            }
            /* the triangle at the end: diagonal d0 + k has N - d0 - k rows */
            for (int k = 0; k < PB_D; ++k) {
                const int64_t d = d0 + k;
                if (d >= N) break;
                const int64_t i_lo = full > 0 ? full : 0;
                if (i_lo + d >= N) continue;
                double c = cov_direct(&s, i_lo, i_lo + d);
                for (int64_t i = i_lo; i + d < N; ++i) {
                    const int64_t j = i + d;
                    double dd = twom * (1.0 - c * iv[i] * iv[j]);
                    dd = dd < 0.0 ? 0.0 : dd;
                    if (dd < mnn[i]) mnn[i] = dd;
                    if (dd < mnn[j]) mnn[j] = dd;
                    if (j + 1 < N) c += df[i] * dg[j] + df[j] * dg[i];
                }
            }
        }
    }
    int64_t flo = -1, fhi = -1;
    for (int64_t i = 0; i < N; ++i)
        if (s.flat[i]) {
            if (flo < 0) flo = i;
            fhi = i;
        }
    for (int64_t i = 0; i < N; ++i) {
        double b = INFINITY;
        for (int t = 0; t < nth; ++t) {
            const double d = tnn[(size_t)t * (N + PB_D) + i];
            if (d < b) b = d;
        }
        if (s.flat[i] && (i - flo >= gap || fhi - i >= gap)) b = 0.0;
        nn[i] = b;
    }
    free(tnn);
    free(df);
    free(dg);
    free(iv);
    series_free(&s);
}

/* nn of many windows (FP64, direct dot products, GPU exclusion rule), in
 * parallel over the windows: out[q] = nn of window w[q], arg[q] its nearest
 * neighbour (lowest index on ties).  Statistics are computed once. */
OR_EXPORT void or_windows_nn(const float *x, int64_t n, int32_t m, const int64_t *w,
                             int64_t count, double *out, int64_t *arg)
{
    or_series s;
    series_init(&s, x, n, m);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < count; ++q) {
        const int64_t i = w[q];
        double best = INFINITY;
        int64_t bj = -1;
        for (int64_t j = 0; j < s.N; ++j) {
            const int64_t dd = i > j ? i - j : j - i;
            if (dd < m - 1) continue;
            const double d = dist_from_cov(&s, i, j, cov_direct(&s, i, j));
            if (d < best) {
                best = d;
                bj = j;
            }
        }
        out[q] = best;
        if (arg) arg[q] = bj;
    }
    series_free(&s);
}

/*
 * out[L] = FP64 nn at length minL + L of window w[L] (one window per length,
 * e.g. the reported top-1 of every length of a PALMAD run), in parallel over
 * the lengths.  The statistics of a length come from long-double window sums
 * slid along blocks of 4096 windows, each block shifted by its own first
 * value (O(N); one prefix over the whole series would accumulate the rounding
 * of ~n squares of the series' full range -- 2e-6 relative on a 2^20-point
 * random walk); flatness is the exact run test.  The dot products are direct
 * and centred on both sides.
 */
OR_EXPORT void or_lengths_nn(const float *x, int64_t n, int32_t minL, int32_t maxL,
                             const int64_t *w, double *out)
{
    const int32_t L = maxL - minL + 1;
    const int64_t B = 4096;
    int64_t *runs = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    runs[n - 1] = 1;
    for (int64_t i = n - 2; i >= 0; --i) runs[i] = (x[i] == x[i + 1]) ? runs[i + 1] + 1 : 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t q = 0; q < L; ++q) {
        const int32_t m = minL + q;
        const int64_t N = n - m + 1;
        const int64_t i = w[q];
        if (i < 0 || i >= N) {
            out[q] = NAN;
            continue;
        }
        double *mu = (double *)malloc(sizeof(double) * (size_t)N);
        double *inv = (double *)malloc(sizeof(double) * (size_t)N);
        uint8_t *fl = (uint8_t *)malloc((size_t)N);
        for (int64_t b0 = 0; b0 < N; b0 += B) {
            const int64_t b1 = b0 + B < N ? b0 + B : N;
            const long double c = (long double)x[b0];
            long double s1 = 0.0L, s2 = 0.0L;
            for (int32_t k = 0; k < m; ++k) {
                const long double d = (long double)x[b0 + k] - c;
                s1 += d;
                s2 += d * d;
            }
            for (int64_t j = b0; j < b1; ++j) {
                const long double u = s1 / m;
                long double v = s2 - s1 * u;
                fl[j] = runs[j] >= m;
                mu[j] = fl[j] ? (double)x[j] : (double)(c + u);
                if (v < 0.0L) v = 0.0L;
                inv[j] = (fl[j] || v == 0.0L) ? 0.0 : (double)(1.0L / sqrtl(v));
                if (inv[j] == 0.0) fl[j] = 1;
                if (j + 1 < b1) { /* slide to window j + 1 */
                    const long double dout = (long double)x[j] - c;
                    const long double din = (long double)x[j + m] - c;
                    s1 += din - dout;
                    s2 += din * din - dout * dout;
                }
            }
        }
        double *a = (double *)malloc(sizeof(double) * (size_t)m);
        for (int32_t k = 0; k < m; ++k) a[k] = (double)x[i + k] - mu[i];
        double best = INFINITY;
        for (int64_t j = 0; j < N; ++j) {
            const int64_t dd = i > j ? i - j : j - i;
            if (dd < m - 1) continue;
            double rho;
            if (fl[i] | fl[j]) {
                rho = (fl[i] & fl[j]) ? 1.0 : 0.0;
            } else {
                const float *b = x + j;
                const double ub = mu[j];
                double acc = 0.0;
                for (int32_t k = 0; k < m; ++k) acc += a[k] * ((double)b[k] - ub);
                rho = acc * inv[i] * inv[j];
            }
            double d = 2.0 * m * (1.0 - rho);
            d = d < 0.0 ? 0.0 : d;
            if (d < best) best = d;
        }
        out[q] = best;
        free(a);
        free(mu);
        free(inv);
        free(fl);
    }
    free(runs);
}

/* nn of a single window (FP64, direct), GPU exclusion rule. */
OR_EXPORT double or_window_nn(const float *x, int64_t n, int32_t m, int64_t i, int64_t *arg)
{
    or_series s;
    series_init(&s, x, n, m);
    double best = INFINITY;
    int64_t bj = -1;
    for (int64_t j = 0; j < s.N; ++j) {
        const int64_t dd = i > j ? i - j : j - i;
        if (dd < m - 1) continue;
        const double d = dist_from_cov(&s, i, j, cov_direct(&s, i, j));
        if (d < best) {
            best = d;
            bj = j;
        }
    }
    series_free(&s);
    if (arg) *arg = bj;
    return best;
}

/* ------------------------------------------------------------------ */
/* selection for one (m, r^2) attempt                                   */
/* ------------------------------------------------------------------ */

typedef struct {
    int32_t ind;
    float dist; /* squared distance, as the reference's Discord (src/PALMAD_types.hpp:7-11) */
} or_discord;

typedef struct {
    int32_t m;
    float r;        /* linear r as the schedule holds it */
    float r2;       /* threshold actually used: r*r in float */
    int64_t n_cand; /* windows never pruned: nn >= r2 */
    int64_t n_disc; /* candidates with nn > r2 (src/sets_processing.hpp:37) */
    int32_t found;  /* 1 if at least top_k discords were selected */
    int32_t n_sel;
    or_discord top; /* best discord or {-1, -FLT_MAX} */
} or_attempt;

/*
 * Given an nn profile (squared distances, FP64) and a threshold r2 (float):
 * candidates = {i : nn_i >= r2} (never pruned by a d < r2 neighbour),
 * discords   = {i : nn_i > r2}  (src/sets_processing.hpp:28,37),
 * selection  = greedy by nn descending, lowest index first on ties, skipping
 *              windows within m-1 of an already selected one
 *              (non_overlap rule of src/PD3_kernels.cuh:70), at most top_k.
 * The comparisons are made on float(nn) against r2, since the reference
 * compares its float nnDist against its float r*r.
 */
OR_EXPORT void or_select(const double *nn, int64_t N, int32_t m, float r2, int32_t top_k,
                         or_attempt *att, or_discord *sel)
{
    int64_t nc = 0, nd = 0;
    for (int64_t i = 0; i < N; ++i) {
        const float f = (float)nn[i];
        nc += f >= r2;
        nd += f > r2;
    }
    att->n_cand = nc;
    att->n_disc = nd;
    att->r2 = r2;
    att->m = m;
    int32_t ns = 0;
    uint8_t *used = (uint8_t *)calloc((size_t)N, 1);
    while (ns < top_k) {
        int64_t b = -1;
        float bd = -FLT_MAX;
        for (int64_t i = 0; i < N; ++i) {
            const float f = (float)nn[i];
            if (used[i] || !(f > r2)) continue;
            if (f > bd) { /* strict: first maximum wins */
                bd = f;
                b = i;
            }
        }
        if (b < 0) break;
        sel[ns].ind = (int32_t)b;
        sel[ns].dist = bd;
        ++ns;
        const int64_t lo = b - (m - 2) < 0 ? 0 : b - (m - 2);
        const int64_t hi = b + (m - 2) >= N ? N - 1 : b + (m - 2);
        for (int64_t i = lo; i <= hi; ++i) used[i] = 1;
        used[b] = 1;
    }
    free(used);
    att->n_sel = ns;
    att->found = ns > 0 && ns >= top_k;
    if (ns > 0) att->top = sel[0];
    else {
        att->top.ind = -1;
        att->top.dist = -FLT_MAX;
    }
}

/* ------------------------------------------------------------------ */
/* schedules                                                            */
/* ------------------------------------------------------------------ */

/* C++ <cmath> overloads the reference relies on: sqrt(float) -> float,
 * pow(float, int) -> double, sqrt(unsigned) -> double. */
static inline float sqrt_f(float v) { return sqrtf(v); }

/*
 * PALMAD over minL..maxL (src/main.cu:136-233), top-1 per length.
 * out[L] = top-1 discord of length minL+L; log receives one row per attempt
 * (at most log_cap rows); returns the number of attempts, or -1 if some
 * length needed more than iter_cap attempts (the reference would loop
 * forever there).
 */
OR_EXPORT int64_t or_palmad(const float *x, int64_t n, int32_t minL, int32_t maxL,
                            int32_t iter_cap, or_discord *out, or_attempt *log,
                            int64_t log_cap, double *nn_out_last)
{
    const int32_t L = maxL - minL + 1;
    int64_t natt = 0;
    for (int32_t j = 0; j < L; ++j) {
        out[j].ind = -1;
        out[j].dist = -FLT_MAX;
    }
    float r = (float)(2.0 * sqrt((double)(unsigned)minL)); /* src/main.cu:38 */
    for (int32_t j = 0; j < L; ++j) {
        const int32_t m = minL + j;
        const int64_t N = n - m + 1;
        double *nn = (double *)malloc(sizeof(double) * (size_t)N);
        int64_t *ix = (int64_t *)malloc(sizeof(int64_t) * (size_t)N);
        or_nn_profile(x, n, m, m - 1, m - 1, 1, nn, ix);
        float S = 0.0f;
        if (j >= 1 && j < 5) {
            r = (float)((double)sqrt_f(out[j - 1].dist) * 0.99); /* src/main.cu:171 */
        } else if (j >= 5) {
            float M = 0.0f;
            for (int k = j - 5; k < j; ++k) M += sqrt_f(out[k].dist); /* :205-206 */
            M = (float)((double)M * 0.2);                              /* :208 */
            for (int k = j - 5; k < j; ++k) {
                const float dv = sqrt_f(out[k].dist) - M;
                S = (float)((double)S + pow((double)dv, 2.0));         /* :210-211 */
            }
            S = (float)sqrt((double)S * 0.2);                          /* :213 */
            r = M - 2 * S;                                             /* :214 */
        }
        int32_t it = 0;
        while (out[j].dist < 0) {
            if (it++ >= iter_cap) {
                free(nn);
                free(ix);
                return -1;
            }
            or_attempt a;
            or_discord sel;
            memset(&a, 0, sizeof(a));
            or_select(nn, N, m, r * r, 1, &a, &sel);
            a.r = r;
            out[j] = a.top;
            if (log && natt < log_cap) log[natt] = a;
            ++natt;
            if (j == 0) r = (float)(0.5 * (double)r);        /* :155 */
            else if (j < 5) r = (float)(0.99 * (double)r);   /* :187 */
            else r = r - S;                                  /* :230 */
        }
        if (nn_out_last && j == L - 1) memcpy(nn_out_last, nn, sizeof(double) * (size_t)N);
        free(nn);
        free(ix);
    }
    return natt;
}

/*
 * Fixed-length discords with top-k: r starts at 2*sqrt(m) and is halved
 * until top_k non-overlapping discords exist (the reference's first-length
 * loop, src/main.cu:136-156, with the top-k condition its comment at :137
 * names).  Returns the number of discords written (<= top_k) and the number
 * of attempts in *n_att; -1 if iter_cap attempts did not suffice.
 */
OR_EXPORT int32_t or_pd3(const float *x, int64_t n, int32_t m, int32_t top_k,
                         int32_t iter_cap, or_discord *sel, or_attempt *log,
                         int64_t log_cap, int64_t *n_att, int32_t fast)
{
    const int64_t N = n - m + 1;
    double *nn = (double *)malloc(sizeof(double) * (size_t)N);
    int64_t *ix = (int64_t *)malloc(sizeof(int64_t) * (size_t)N);
    /* fast: the vectorised profile re-anchored every 8192 rows (long series) */
    if (fast) or_nn_profile_fast(x, n, m, nn);
    else or_nn_profile(x, n, m, m - 1, m - 1, 1, nn, ix);
    float r = (float)(2.0 * sqrt((double)(unsigned)m));
    int64_t na = 0;
    int32_t ns = 0;
    for (;;) {
        if (na >= iter_cap) {
            ns = -1;
            break;
        }
        or_attempt a;
        memset(&a, 0, sizeof(a));
        or_select(nn, N, m, r * r, top_k, &a, sel);
        a.r = r;
        if (log && na < log_cap) log[na] = a;
        ++na;
        if (a.found || r * r == 0.0f) { /* r^2 == 0 admits every nn > 0 */
            ns = a.n_sel;
            break;
        }
        r = (float)(0.5 * (double)r);
    }
    *n_att = na;
    free(nn);
    free(ix);
    return ns;
}
