/*
 * oracle.c -- CPU oracle for the GEMM path. TEST INFRASTRUCTURE ONLY (see
 * oracle.h). Only tests/, the smoke check and bench.py's CPU-baseline leg load
 * this file's library, and only to check results.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NOTRANS 111
#define TRANS 112
#define CONJTRANS 113

/* ------------------------------------------------------------------------ */
/* Tiled restatement of the reference algorithm                              */
/* ------------------------------------------------------------------------ */

/* Edge-tile clipping, following margin_adjustment (blas/blasx_mem_control.c:24-42):
 * the tile on the last block row/column holds the residual rows/columns. The
 * reference computes its grid bounds so that an exact multiple never reaches
 * the residual branch (blas/blasx_dgemm.c:284-296); the same holds here. */
static void margin(int nrow, int ncol, int bd, int br, int bc, int *r, int *c) {
    *r = (br == nrow / bd) ? nrow % bd : bd;
    *c = (bc == ncol / bd) ? ncol % bd : bd;
}

/* Number of block rows/cols - 1, as x/y/z in blas/blasx_dgemm.c:284-296. */
static int last_block(int n, int bd) { return (n % bd == 0) ? n / bd - 1 : n / bd; }

#define TILED_BODY(T, ACC_T, MUL_ADD)                                                        \
    int nrowa = (transa == NOTRANS) ? M : K, ncola = (transa == NOTRANS) ? K : M;            \
    int nrowb = (transb == NOTRANS) ? K : N, ncolb = (transb == NOTRANS) ? N : K;            \
    (void)ncola; (void)nrowb;                                                                \
    int x = last_block(M, bd), y = last_block(N, bd);                                        \
    int z = last_block(K, bd);                                                               \
    (void)nrowa; (void)ncolb;                                                                \
    /* one task per C tile, t -> (i = t/(y+1), k = t%(y+1)) (blas/blasx_dgemm.c:28-29) */    \
    for (int t = 0; t <= (x + 1) * (y + 1) - 1; ++t) {                                       \
        int i = t / (y + 1), k = t % (y + 1);                                                \
        int mr, nc;                                                                          \
        margin(M, N, bd, i, k, &mr, &nc);                                                    \
        for (int j = 0; j <= z; ++j) {                                                       \
            int kr, kc;                                                                      \
            margin(K, K, bd, j, j, &kr, &kc);                                                \
            (void)kc;                                                                        \
            /* beta on the first K-step, 1 afterwards (blas/blasx_dgemm.c:82) */             \
            int first = (j == 0);                                                            \
            for (int c = 0; c < nc; ++c) {                                                   \
                for (int r = 0; r < mr; ++r) {                                               \
                    long gi = (long)i * bd + r, gj = (long)k * bd + c;                       \
                    ACC_T s = 0;                                                             \
                    for (int q = 0; q < kr; ++q) {                                           \
                        long gk = (long)j * bd + q;                                          \
                        MUL_ADD                                                              \
                    }                                                                        \
                    T *cp = &C[gi + gj * (long)ldc];                                         \
                    STORE                                                                    \
                }                                                                            \
            }                                                                                \
        }                                                                                    \
    }

static inline double getA_d(const double *A, int lda, int tr, long i, long k) {
    return tr == NOTRANS ? A[i + k * (long)lda] : A[k + i * (long)lda];
}
static inline double getB_d(const double *B, int ldb, int tr, long k, long j) {
    return tr == NOTRANS ? B[k + j * (long)ldb] : B[j + k * (long)ldb];
}
static inline float getA_s(const float *A, int lda, int tr, long i, long k) {
    return tr == NOTRANS ? A[i + k * (long)lda] : A[k + i * (long)lda];
}
static inline float getB_s(const float *B, int ldb, int tr, long k, long j) {
    return tr == NOTRANS ? B[k + j * (long)ldb] : B[j + k * (long)ldb];
}

void oracle_dgemm_tiled(int transa, int transb, int M, int N, int K, double alpha,
                        const double *A, int lda, const double *B, int ldb, double beta,
                        double *C, int ldc, int bd) {
    if (M <= 0 || N <= 0) return;
    if (K <= 0 || alpha == 0) { /* C <- beta C: A, B not read; C not read when beta == 0 */
        for (int c = 0; c < N; ++c)
            for (int r = 0; r < M; ++r)
                C[r + (long)c * ldc] = beta == 0 ? 0.0 : beta * C[r + (long)c * ldc];
        return;
    }
#define STORE *cp = first ? (beta == 0 ? alpha * s : alpha * s + beta * *cp) : alpha * s + *cp;
    TILED_BODY(double, double,
               s = fma(getA_d(A, lda, transa, gi, gk), getB_d(B, ldb, transb, gk, gj), s);)
#undef STORE
}

void oracle_sgemm_tiled(int transa, int transb, int M, int N, int K, float alpha,
                        const float *A, int lda, const float *B, int ldb, float beta,
                        float *C, int ldc, int bd) {
    if (M <= 0 || N <= 0) return;
    if (K <= 0 || alpha == 0) {
        for (int c = 0; c < N; ++c)
            for (int r = 0; r < M; ++r)
                C[r + (long)c * ldc] = beta == 0 ? 0.0f : beta * C[r + (long)c * ldc];
        return;
    }
#define STORE *cp = first ? (beta == 0 ? alpha * s : alpha * s + beta * *cp) : alpha * s + *cp;
    TILED_BODY(float, float,
               s = fmaf(getA_s(A, lda, transa, gi, gk), getB_s(B, ldb, transb, gk, gj), s);)
#undef STORE
}

/* complex helpers: element (re, im) of op(A) at (i, k) */
static inline void getA_z(const double *A, int lda, int tr, long i, long k, double *re, double *im) {
    const double *p = tr == NOTRANS ? &A[2 * (i + k * (long)lda)] : &A[2 * (k + i * (long)lda)];
    *re = p[0];
    *im = tr == CONJTRANS ? -p[1] : p[1];
}
static inline void getB_z(const double *B, int ldb, int tr, long k, long j, double *re, double *im) {
    const double *p = tr == NOTRANS ? &B[2 * (k + j * (long)ldb)] : &B[2 * (j + k * (long)ldb)];
    *re = p[0];
    *im = tr == CONJTRANS ? -p[1] : p[1];
}

void oracle_zgemm_tiled(int transa, int transb, int M, int N, int K, const double *alpha,
                        const double *A, int lda, const double *B, int ldb, const double *beta,
                        double *C, int ldc, int bd) {
    if (M <= 0 || N <= 0) return;
    double ar = alpha[0], ai = alpha[1], br_ = beta[0], bi_ = beta[1];
    int beta_zero = (br_ == 0 && bi_ == 0);
    if (K <= 0 || (ar == 0 && ai == 0)) {
        for (int c = 0; c < N; ++c)
            for (int r = 0; r < M; ++r) {
                double *p = &C[2 * (r + (long)c * ldc)];
                if (beta_zero) { p[0] = 0; p[1] = 0; continue; }
                double re = br_ * p[0] - bi_ * p[1], im = br_ * p[1] + bi_ * p[0];
                p[0] = re; p[1] = im;
            }
        return;
    }
    int x = last_block(M, bd), y = last_block(N, bd), z = last_block(K, bd);
    for (int t = 0; t <= (x + 1) * (y + 1) - 1; ++t) {
        int i = t / (y + 1), k = t % (y + 1);
        int mr, nc;
        margin(M, N, bd, i, k, &mr, &nc);
        for (int j = 0; j <= z; ++j) {
            int kr, kc;
            margin(K, K, bd, j, j, &kr, &kc);
            (void)kc;
            int first = (j == 0);
            for (int c = 0; c < nc; ++c)
                for (int r = 0; r < mr; ++r) {
                    long gi = (long)i * bd + r, gj = (long)k * bd + c;
                    double sr = 0, si = 0;
                    for (int q = 0; q < kr; ++q) {
                        long gk = (long)j * bd + q;
                        double xr, xi, yr, yi;
                        getA_z(A, lda, transa, gi, gk, &xr, &xi);
                        getB_z(B, ldb, transb, gk, gj, &yr, &yi);
                        sr = fma(xr, yr, sr); sr = fma(-xi, yi, sr);
                        si = fma(xr, yi, si); si = fma(xi, yr, si);
                    }
                    double *p = &C[2 * (gi + gj * (long)ldc)];
                    double tr = ar * sr - ai * si, ti = ar * si + ai * sr;
                    if (first) {
                        if (!beta_zero) {
                            tr += br_ * p[0] - bi_ * p[1];
                            ti += br_ * p[1] + bi_ * p[0];
                        }
                    } else {
                        tr += p[0];
                        ti += p[1];
                    }
                    p[0] = tr; p[1] = ti;
                }
        }
    }
}

/* complex64: the same tiled algorithm in float arithmetic (the precision of
 * the reference's CPU cblas_cgemm, blas/cgemm.c:60-68) */
static inline void getA_c(const float *A, int lda, int tr, long i, long k, float *re, float *im) {
    const float *p = tr == NOTRANS ? &A[2 * (i + k * (long)lda)] : &A[2 * (k + i * (long)lda)];
    *re = p[0];
    *im = tr == CONJTRANS ? -p[1] : p[1];
}
static inline void getB_c(const float *B, int ldb, int tr, long k, long j, float *re, float *im) {
    const float *p = tr == NOTRANS ? &B[2 * (k + j * (long)ldb)] : &B[2 * (j + k * (long)ldb)];
    *re = p[0];
    *im = tr == CONJTRANS ? -p[1] : p[1];
}

void oracle_cgemm_tiled(int transa, int transb, int M, int N, int K, const float *alpha,
                        const float *A, int lda, const float *B, int ldb, const float *beta,
                        float *C, int ldc, int bd) {
    if (M <= 0 || N <= 0) return;
    float ar = alpha[0], ai = alpha[1], br_ = beta[0], bi_ = beta[1];
    int beta_zero = (br_ == 0 && bi_ == 0);
    if (K <= 0 || (ar == 0 && ai == 0)) {
        for (int c = 0; c < N; ++c)
            for (int r = 0; r < M; ++r) {
                float *p = &C[2 * (r + (long)c * ldc)];
                if (beta_zero) { p[0] = 0; p[1] = 0; continue; }
                float re = br_ * p[0] - bi_ * p[1], im = br_ * p[1] + bi_ * p[0];
                p[0] = re; p[1] = im;
            }
        return;
    }
    int x = last_block(M, bd), y = last_block(N, bd), z = last_block(K, bd);
    for (int t = 0; t <= (x + 1) * (y + 1) - 1; ++t) {
        int i = t / (y + 1), k = t % (y + 1);
        int mr, nc;
        margin(M, N, bd, i, k, &mr, &nc);
        for (int j = 0; j <= z; ++j) {
            int kr, kc;
            margin(K, K, bd, j, j, &kr, &kc);
            (void)kc;
            int first = (j == 0);
            for (int c = 0; c < nc; ++c)
                for (int r = 0; r < mr; ++r) {
                    long gi = (long)i * bd + r, gj = (long)k * bd + c;
                    float sr = 0, si = 0;
                    for (int q = 0; q < kr; ++q) {
                        long gk = (long)j * bd + q;
                        float xr, xi, yr, yi;
                        getA_c(A, lda, transa, gi, gk, &xr, &xi);
                        getB_c(B, ldb, transb, gk, gj, &yr, &yi);
                        sr = fmaf(xr, yr, sr); sr = fmaf(-xi, yi, sr);
                        si = fmaf(xr, yi, si); si = fmaf(xi, yr, si);
                    }
                    float *p = &C[2 * (gi + gj * (long)ldc)];
                    float tr = ar * sr - ai * si, ti = ar * si + ai * sr;
                    if (first) {
                        if (!beta_zero) {
                            tr += br_ * p[0] - bi_ * p[1];
                            ti += br_ * p[1] + bi_ * p[0];
                        }
                    } else {
                        tr += p[0];
                        ti += p[1];
                    }
                    p[0] = tr; p[1] = ti;
                }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Double-double sampled-entry oracle (Ogita-Rump-Oishi Dot2)                */
/* ------------------------------------------------------------------------ */

typedef struct { double hi, lo; } dd;

static inline void two_sum(double a, double b, double *s, double *e) {
    double x = a + b, z = x - a;
    *s = x;
    *e = (a - (x - z)) + (b - z);
}
static inline void two_prod(double a, double b, double *p, double *e) {
    double x = a * b;
    *p = x;
    *e = fma(a, b, -x);
}
/* Dot2 accumulator: p accumulates the rounded sum, s the error terms. */
typedef struct { double p, s; } dot2;
static inline void dot2_add_prod(dot2 *d, double a, double b) {
    double h, r, q;
    two_prod(a, b, &h, &r);
    two_sum(d->p, h, &d->p, &q);
    d->s += q + r;
}
static inline void dot2_add(dot2 *d, double a) {
    double q;
    two_sum(d->p, a, &d->p, &q);
    d->s += q;
}
static inline dd dot2_result(dot2 d) {
    dd o;
    two_sum(d.p, d.s, &o.hi, &o.lo);
    return o;
}
/* multiply a dot2 value by a double scalar, returning a fresh accumulator */
static inline dot2 dot2_scale(dot2 d, double a) {
    dot2 o = {0, 0};
    dd v = dot2_result(d);
    dot2_add_prod(&o, v.hi, a);
    dot2_add_prod(&o, v.lo, a);
    return o;
}

void oracle_dgemm_dd_entries(int transa, int transb, int M, int N, int K, double alpha,
                             const double *A, int lda, const double *B, int ldb, double beta,
                             const double *C0, int ldc, int64_t n, const int64_t *ii,
                             const int64_t *jj, double *hi, double *lo, double *bound) {
    (void)M; (void)N;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < n; ++t) {
        long i = ii[t], j = jj[t];
        dot2 d = {0, 0};
        double absum = 0;
        for (long q = 0; q < K; ++q) {
            double a = getA_d(A, lda, transa, i, q), b = getB_d(B, ldb, transb, q, j);
            dot2_add_prod(&d, a, b);
            absum += fabs(a) * fabs(b);
        }
        dot2 r = dot2_scale(d, alpha);
        double bnd = fabs(alpha) * absum;
        if (beta != 0 && C0) {
            double c = C0[i + j * (long)ldc];
            dot2_add_prod(&r, beta, c);
            bnd += fabs(beta) * fabs(c);
        }
        dd v = dot2_result(r);
        hi[t] = v.hi; lo[t] = v.lo; bound[t] = bnd;
    }
}

void oracle_sgemm_dd_entries(int transa, int transb, int M, int N, int K, float alpha,
                             const float *A, int lda, const float *B, int ldb, float beta,
                             const float *C0, int ldc, int64_t n, const int64_t *ii,
                             const int64_t *jj, double *hi, double *lo, double *bound) {
    (void)M; (void)N;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < n; ++t) {
        long i = ii[t], j = jj[t];
        dot2 d = {0, 0};
        double absum = 0;
        for (long q = 0; q < K; ++q) {
            double a = getA_s(A, lda, transa, i, q), b = getB_s(B, ldb, transb, q, j);
            dot2_add_prod(&d, a, b); /* exact: float*float fits in double */
            absum += fabs(a) * fabs(b);
        }
        dot2 r = dot2_scale(d, (double)alpha);
        double bnd = fabs((double)alpha) * absum;
        if (beta != 0 && C0) {
            double c = C0[i + j * (long)ldc];
            dot2_add_prod(&r, (double)beta, c);
            bnd += fabs((double)beta) * fabs(c);
        }
        dd v = dot2_result(r);
        hi[t] = v.hi; lo[t] = v.lo; bound[t] = bnd;
    }
}

void oracle_zgemm_dd_entries(int transa, int transb, int M, int N, int K, const double *alpha,
                             const double *A, int lda, const double *B, int ldb,
                             const double *beta, const double *C0, int ldc, int64_t n,
                             const int64_t *ii, const int64_t *jj, double *hi, double *lo,
                             double *bound) {
    (void)M; (void)N;
    int beta_zero = beta[0] == 0 && beta[1] == 0;
    double aabs = hypot(alpha[0], alpha[1]), babs = hypot(beta[0], beta[1]);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < n; ++t) {
        long i = ii[t], j = jj[t];
        dot2 re = {0, 0}, im = {0, 0};
        double absum = 0;
        for (long q = 0; q < K; ++q) {
            double xr, xi, yr, yi;
            getA_z(A, lda, transa, i, q, &xr, &xi);
            getB_z(B, ldb, transb, q, j, &yr, &yi);
            dot2_add_prod(&re, xr, yr);
            dot2_add_prod(&re, -xi, yi);
            dot2_add_prod(&im, xr, yi);
            dot2_add_prod(&im, xi, yr);
            absum += hypot(xr, xi) * hypot(yr, yi);
        }
        /* (alpha_r + i alpha_i)(re + i im) */
        dd vr = dot2_result(re), vi = dot2_result(im);
        dot2 orr = {0, 0}, oi = {0, 0};
        dot2_add_prod(&orr, alpha[0], vr.hi); dot2_add_prod(&orr, alpha[0], vr.lo);
        dot2_add_prod(&orr, -alpha[1], vi.hi); dot2_add_prod(&orr, -alpha[1], vi.lo);
        dot2_add_prod(&oi, alpha[0], vi.hi); dot2_add_prod(&oi, alpha[0], vi.lo);
        dot2_add_prod(&oi, alpha[1], vr.hi); dot2_add_prod(&oi, alpha[1], vr.lo);
        double bnd = aabs * absum;
        if (!beta_zero && C0) {
            const double *c = &C0[2 * (i + j * (long)ldc)];
            dot2_add_prod(&orr, beta[0], c[0]); dot2_add_prod(&orr, -beta[1], c[1]);
            dot2_add_prod(&oi, beta[0], c[1]); dot2_add_prod(&oi, beta[1], c[0]);
            bnd += babs * hypot(c[0], c[1]);
        }
        dd a = dot2_result(orr), b = dot2_result(oi);
        hi[2 * t] = a.hi; lo[2 * t] = a.lo;
        hi[2 * t + 1] = b.hi; lo[2 * t + 1] = b.lo;
        bound[2 * t] = bnd; bound[2 * t + 1] = bnd;
        (void)dot2_add;
    }
}

/* ------------------------------------------------------------------------ */
/* OpenBLAS via dlopen                                                       */
/* ------------------------------------------------------------------------ */

typedef void (*dgemm32_t)(int, int, int, int, int, int, double, const double *, int,
                          const double *, int, double, double *, int);
typedef void (*sgemm32_t)(int, int, int, int, int, int, float, const float *, int,
                          const float *, int, float, float *, int);
typedef void (*zgemm32_t)(int, int, int, int, int, int, const void *, const void *, int,
                          const void *, int, const void *, void *, int);
typedef void (*dgemm64_t)(int, int, int, int64_t, int64_t, int64_t, double, const double *,
                          int64_t, const double *, int64_t, double, double *, int64_t);
typedef void (*sgemm64_t)(int, int, int, int64_t, int64_t, int64_t, float, const float *,
                          int64_t, const float *, int64_t, float, float *, int64_t);
typedef void (*zgemm64_t)(int, int, int, int64_t, int64_t, int64_t, const void *, const void *,
                          int64_t, const void *, int64_t, const void *, void *, int64_t);

static void *g_blas;
static int g_ilp64;
static void *g_d, *g_s, *g_z, *g_c;
static char g_name[1024];

int oracle_openblas_open(const char *paths) {
    if (g_blas) return 0;
    char *buf = strdup(paths), *save = NULL;
    for (char *tok = strtok_r(buf, ":", &save); tok; tok = strtok_r(NULL, ":", &save)) {
        char *bar1 = strchr(tok, '|');
        if (!bar1) continue;
        *bar1 = 0;
        char *prefix = bar1 + 1, *bar2 = strchr(prefix, '|');
        if (!bar2) continue;
        *bar2 = 0;
        int ilp = atoi(bar2 + 1);
        void *h = dlopen(tok, RTLD_NOW | RTLD_LOCAL);
        if (!h) continue;
        char sym[256];
        const char *suffix = ilp ? "64_" : "";
        snprintf(sym, sizeof sym, "%scblas_dgemm%s", prefix, suffix);
        void *d = dlsym(h, sym);
        snprintf(sym, sizeof sym, "%scblas_sgemm%s", prefix, suffix);
        void *s = dlsym(h, sym);
        snprintf(sym, sizeof sym, "%scblas_zgemm%s", prefix, suffix);
        void *z = dlsym(h, sym);
        snprintf(sym, sizeof sym, "%scblas_cgemm%s", prefix, suffix);
        void *cg = dlsym(h, sym);
        if (!d || !s || !z) { dlclose(h); continue; }
        g_blas = h; g_d = d; g_s = s; g_z = z; g_c = cg; g_ilp64 = ilp;
        char ver[128] = "";
        char vsym[256];
        snprintf(vsym, sizeof vsym, "%sopenblas_get_config%s", prefix, ilp ? "64_" : "");
        const char *(*cfg)(void) = (const char *(*)(void))dlsym(h, vsym);
        if (cfg) snprintf(ver, sizeof ver, "%s", cfg());
        snprintf(g_name, sizeof g_name, "%s [%s%s] %s", tok, prefix, ilp ? " ilp64" : "", ver);
        free(buf);
        return 0;
    }
    free(buf);
    return -1;
}

const char *oracle_openblas_name(void) { return g_blas ? g_name : ""; }

int oracle_openblas_dgemm(int order, int transa, int transb, int M, int N, int K, double alpha,
                          const double *A, int lda, const double *B, int ldb, double beta,
                          double *C, int ldc) {
    if (!g_blas) return -1;
    if (g_ilp64)
        ((dgemm64_t)g_d)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
        ((dgemm32_t)g_d)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return 0;
}

int oracle_openblas_sgemm(int order, int transa, int transb, int M, int N, int K, float alpha,
                          const float *A, int lda, const float *B, int ldb, float beta,
                          float *C, int ldc) {
    if (!g_blas) return -1;
    if (g_ilp64)
        ((sgemm64_t)g_s)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
        ((sgemm32_t)g_s)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return 0;
}

int oracle_openblas_cgemm(int order, int transa, int transb, int M, int N, int K,
                          const float *alpha, const float *A, int lda, const float *B,
                          int ldb, const float *beta, float *C, int ldc) {
    if (!g_blas || !g_c) return -1;
    if (g_ilp64)
        ((zgemm64_t)g_c)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
        ((zgemm32_t)g_c)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return 0;
}

int oracle_openblas_zgemm(int order, int transa, int transb, int M, int N, int K,
                          const double *alpha, const double *A, int lda, const double *B,
                          int ldb, const double *beta, double *C, int ldc) {
    if (!g_blas) return -1;
    if (g_ilp64)
        ((zgemm64_t)g_z)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
        ((zgemm32_t)g_z)(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Seeded generators                                                         */
/* ------------------------------------------------------------------------ */

static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
static inline double u01(uint64_t seed, uint64_t t) {
    return (double)(splitmix64(seed * 0x100000001B3ull ^ t) >> 11) * 0x1.0p-53;
}

void oracle_fill_uniform_f64(double *x, int64_t n, uint64_t seed, double lo, double hi) {
    for (int64_t t = 0; t < n; ++t) x[t] = lo + (hi - lo) * u01(seed, (uint64_t)t);
}
void oracle_fill_uniform_f32(float *x, int64_t n, uint64_t seed, float lo, float hi) {
    for (int64_t t = 0; t < n; ++t) x[t] = (float)(lo + (hi - lo) * u01(seed, (uint64_t)t));
}
void oracle_fill_spread_f64(double *x, int64_t n, uint64_t seed, double phi) {
    const double two_pi = 6.283185307179586476925286766559;
    for (int64_t t = 0; t < n; ++t) {
        double u = u01(seed, (uint64_t)t) - 0.5;
        double u1 = u01(seed ^ 0x5DEECE66Dull, 2 * (uint64_t)t);
        double u2 = u01(seed ^ 0x5DEECE66Dull, 2 * (uint64_t)t + 1);
        if (u1 < 0x1.0p-60) u1 = 0x1.0p-60;
        double g = sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
        x[t] = u * exp(phi * g);
    }
}
