/*
 * kgwas_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference kgwas 1-D association test, used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker.  Nothing in the product links or calls this file.
 *
 * Parity pin: checked against the reference's own black-box kgwas binary
 * (COLS and ROWS modes) on the golden vectors under tests/golden/.
 *
 * Each step follows the reference literally, in FP64 with long-double
 * accumulation for every dot product (so the oracle is at least as accurate
 * as the reference's FP64 ROWS mode):
 *   - Pearson pre-filter:  src/kgwas.cpp:461-468 (ROWS, FP64) and
 *                          src/kgwas.cpp:182-218 (COLS, same formula in FP32)
 *   - low-rank statistics: src/kgwas.cpp:471-474 (ROWS) / :138-166 (COLS)
 *   - yyM:                 src/kgwas_utils.hpp:151-153
 *   - compute_hit:         src/kgwas.cpp:44-56
 *   - 1-df tail:           src/chisq.hpp:6-9
 *
 * Input layout: x is k-mer-major, wpk uint64 words per k-mer, overlap sample
 * i in bit (i % 64) of word (i / 64).  U is n x k column-major (U.bin body).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef long double ld;

/* -log10 of erfc(sqrt(T/2)) without underflow.  erfcl covers T up to about
 * 2.2e4; beyond that the asymptotic expansion of erfc is used. */
static double mlog10_chi2_sf_k1(double T) {
    if (!(T > 0.0)) return 0.0;
    ld z = sqrtl(0.5L * (ld)T);
    if (T < 20000.0) {
        ld p = erfcl(z);
        if (p > 0.0L) return (double)(-log10l(p));
    }
    /* erfc(z) = exp(-z^2)/(z sqrt(pi)) * (1 - 1/(2z^2) + 3/(4z^4) - 15/(8z^6)) */
    ld iz2 = 1.0L / (z * z);
    ld series = 1.0L - 0.5L * iz2 + 0.75L * iz2 * iz2 - 1.875L * iz2 * iz2 * iz2;
    ld lnp = -z * z - logl(z) - 0.5L * logl(3.14159265358979323846264338327950288L) + logl(series);
    return (double)(-lnp / logl(10.0L));
}

/* compute_hit, src/kgwas.cpp:44-56 */
static void compute_hit(double xxM, double xyM, double yyM, int n,
                        double* effect, double* T, double* pval) {
    const double eps = 1e-12;
    *effect = 0.0; *T = 0.0; *pval = 1.0;
    if (xxM > eps && yyM > eps) {
        double r2 = (xyM * xyM) / (xxM * yyM);
        if (r2 < 0) r2 = 0;
        if (r2 >= 1) r2 = 1 - 1e-15;
        *T = (double)n * log(1.0 / (1.0 - r2));
        *pval = erfc(sqrt(0.5 * *T));
        *effect = xyM / (xxM * yyM);
    }
}

/* yyM = ||y||^2 - ||U^T y||^2 (src/kgwas_utils.hpp:151-153).  Returns yyM and
 * writes U^T y into Uy (length k). */
double kgo_yyM(int n, const double* U, int k, const double* y, double* Uy) {
    ld yy = 0;
    for (int i = 0; i < n; ++i) yy += (ld)y[i] * y[i];
    ld s = 0;
    for (int j = 0; j < k; ++j) {
        ld a = 0;
        const double* u = U + (size_t)j * n;
        for (int i = 0; i < n; ++i) a += (ld)u[i] * y[i];
        if (Uy) Uy[j] = (double)a;
        s += a * a;
    }
    return (double)(yy - s);
}

/*
 * Per-k-mer statistics for one phenotype.  Any output pointer may be NULL.
 *   tested[j]  1 if k-mer j passed the pre-filter (counted in .count)
 *   cor[j]     Pearson correlation (0 for constant columns)
 *   xxM, xyM   low-rank residual products (0 when not tested)
 *   T, pval, effect, mlog10p   compute_hit outputs (1/0 defaults when not tested)
 * Returns the number of tested k-mers.
 */
int64_t kgo_cols(const uint64_t* x, int64_t m, int wpk, int n,
                 const double* U, int k, const double* y, double corr_thr,
                 uint8_t* tested, double* cor_out, double* xxM_out, double* xyM_out,
                 double* T_out, double* p_out, double* eff_out, double* ml_out) {
    double* Uy = (double*)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1));
    const double yyM = kgo_yyM(n, U, k, y, Uy);
    ld ysum = 0;
    for (int i = 0; i < n; ++i) ysum += y[i];
    const ld ymean = ysum / n;
    double* yc = (double*)malloc(sizeof(double) * (size_t)n);
    ld yn = 0;
    for (int i = 0; i < n; ++i) { yc[i] = (double)((ld)y[i] - ymean); yn += (ld)yc[i] * yc[i]; }
    const double ynorm = (double)sqrtl(yn);
    ld* Ux = (ld*)malloc(sizeof(ld) * (size_t)(k > 0 ? k : 1));
    int64_t n_tested = 0;

    for (int64_t j = 0; j < m; ++j) {
        const uint64_t* row = x + (size_t)j * wpk;
        int c = 0;
        for (int w = 0; w < wpk; ++w) c += __builtin_popcountll(row[w]);
        /* x_centered = x - mean(x); its norm and dot with y_centered */
        const ld xm = (ld)c / n;
        ld xn = 0, xy = 0;
        for (int i = 0; i < n; ++i) {
            const int b = (int)((row[i >> 6] >> (i & 63)) & 1u);
            const ld xc = (ld)b - xm;
            xn += xc * xc;
            xy += xc * (ld)yc[i];
        }
        const double xnorm = (double)sqrtl(xn);
        uint8_t pass = 0;
        double cor = 0.0;
        if (!(xnorm < 1e-12 || ynorm < 1e-12)) {
            cor = (double)(xy / ((ld)xnorm * (ld)ynorm));
            if (!(fabs(cor) < corr_thr)) pass = 1;
        }
        double xxM = 0, xyM = 0, eff = 0, T = 0, p = 1, ml = 0;
        if (pass) {
            ++n_tested;
            for (int t = 0; t < k; ++t) Ux[t] = 0;
            ld xdy = 0;
            for (int i = 0; i < n; ++i) {
                if (!((row[i >> 6] >> (i & 63)) & 1u)) continue;
                xdy += y[i];
                for (int t = 0; t < k; ++t) Ux[t] += U[(size_t)t * n + i];
            }
            ld sUX = 0, UyUX = 0;
            for (int t = 0; t < k; ++t) { sUX += Ux[t] * Ux[t]; UyUX += Ux[t] * (ld)Uy[t]; }
            xxM = (double)((ld)c - sUX);
            xyM = (double)(xdy - UyUX);
            compute_hit(xxM, xyM, yyM, n, &eff, &T, &p);
            ml = mlog10_chi2_sf_k1(T);
        }
        if (tested) tested[j] = pass;
        if (cor_out) cor_out[j] = cor;
        if (xxM_out) xxM_out[j] = xxM;
        if (xyM_out) xyM_out[j] = xyM;
        if (T_out) T_out[j] = T;
        if (p_out) p_out[j] = p;
        if (eff_out) eff_out[j] = eff;
        if (ml_out) ml_out[j] = ml;
    }
    free(Ux); free(yc); free(Uy);
    return n_tested;
}

/* -log10 p for an array of chi-square values (same tail as kgo_cols). */
void kgo_mlog10p(const double* T, int64_t m, double* out) {
    for (int64_t j = 0; j < m; ++j) out[j] = mlog10_chi2_sf_k1(T[j]);
}

/*
 * 2-D pair test (src/kgwas_2d.cpp:237-331, emit_pairs_self): for every pair
 * i < j of k-mers with row_start <= i < row_end, the column x12 = x_i * x_j
 * (AND of the packed rows) goes through the same low-rank statistic as one
 * k-mer of the 1-D test, without the Pearson pre-filter:
 *   a33 = popcount(x12) must be > 0 (this implies a11, a22 > 0);
 *   xxM = a33 - ||U^T x12||^2, xyM = x12.y - (U^T x12).(U^T y);
 *   compute_hit (src/kgwas.cpp:44-56).
 * The reference evaluates x12.y and U^T x12 in FP32 (src/kgwas_2d.cpp:306-312);
 * here in long double.  Outputs are dense N x N arrays indexed i*N + j (only
 * i < j inside the row range are written); evaluated[i*N+j] = 1 when a33 > 0,
 * xxM > eps and yyM > eps, the pairs the reference gives a p-value (the
 * others are skipped, src/kgwas_2d.cpp:300-313).  Returns their number.
 */
int64_t kgo_pairs(const uint64_t* x, int64_t N, int wpk, int n, const double* U, int k, const double* y,
                  int64_t row_start, int64_t row_end, uint8_t* evaluated, double* T_out, double* p_out,
                  double* eff_out, double* ml_out) {
    double* Uy = (double*)malloc(sizeof(double) * (size_t)(k > 0 ? k : 1));
    const double yyM = kgo_yyM(n, U, k, y, Uy);
    ld* Ux = (ld*)malloc(sizeof(ld) * (size_t)(k > 0 ? k : 1));
    uint64_t* w12 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)wpk);
    int64_t n_eval = 0;
    if (row_end > N) row_end = N;
    for (int64_t i = row_start; i < row_end; ++i) {
        const uint64_t* xi = x + (size_t)i * wpk;
        for (int64_t j = i + 1; j < N; ++j) {
            const uint64_t* xj = x + (size_t)j * wpk;
            int c = 0;
            for (int w = 0; w < wpk; ++w) { w12[w] = xi[w] & xj[w]; c += __builtin_popcountll(w12[w]); }
            const size_t o = (size_t)i * (size_t)N + (size_t)j;
            double eff = 0, T = 0, p = 1, ml = 0;
            int ev = 0;
            if (c > 0) {
                for (int t = 0; t < k; ++t) Ux[t] = 0;
                ld xdy = 0;
                for (int s = 0; s < n; ++s) {
                    if (!((w12[s >> 6] >> (s & 63)) & 1u)) continue;
                    xdy += y[s];
                    for (int t = 0; t < k; ++t) Ux[t] += U[(size_t)t * n + s];
                }
                ld sUX = 0, UyUX = 0;
                for (int t = 0; t < k; ++t) { sUX += Ux[t] * Ux[t]; UyUX += Ux[t] * (ld)Uy[t]; }
                const double xxM = (double)((ld)c - sUX);
                const double xyM = (double)(xdy - UyUX);
                ev = xxM > 1e-12 && yyM > 1e-12;
                n_eval += ev;
                compute_hit(xxM, xyM, yyM, n, &eff, &T, &p);
                ml = mlog10_chi2_sf_k1(T);
            }
            if (evaluated) evaluated[o] = (uint8_t)ev;
            if (T_out) T_out[o] = T;
            if (p_out) p_out[o] = p;
            if (eff_out) eff_out[o] = eff;
            if (ml_out) ml_out[o] = ml;
        }
    }
    free(w12); free(Ux); free(Uy);
    return n_eval;
}
