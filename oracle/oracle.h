/*
 * oracle.h -- CPU oracle for the GEMM path. TEST INFRASTRUCTURE ONLY.
 *
 * Nothing in the shipped library links or calls this code. It is used by the
 * test-suite, by the smoke check and by bench.py's CPU-baseline leg, always as
 * a check of results and never as the thing that is measured or shipped.
 *
 * Contents:
 *   - oracle_?gemm_tiled: a plain-C restatement of the reference's tiled GEMM
 *     algorithm (blas/blasx_dgemm.c:251-356 tile grid, :5-96 per-tile step
 *     with beta on the first K-step and 1 afterwards, margin_adjustment
 *     blas/blasx_mem_control.c:24-42). The per-tile product that the
 *     reference hands to cuBLAS is a straightforward loop here.
 *   - oracle_?gemm_dd_entries: a compensated (double-double) dot product for
 *     sampled C entries, Ogita-Rump-Oishi "Accurate sum and dot product"
 *     (SIAM J. Sci. Comput. 2005), algorithm Dot2 with FMA-based TwoProduct.
 *     It also returns the componentwise bound scale |alpha||A||B| + |beta||C0|.
 *   - oracle_openblas_*: OpenBLAS resolved at run time with dlopen, the CPU
 *     BLAS the reference dispatches small calls to (blas/blasx_internal.c:26-36).
 *
 * Parity is pinned by tests/golden (outputs of the reference library itself,
 * compiled from its own sources into oracle/_ref, on its CPU path).
 */
#ifndef BLASX_ORACLE_H
#define BLASX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* trans: 111 NoTrans, 112 Trans, 113 ConjTrans (CBLAS enum values). Column-major. */
void oracle_dgemm_tiled(int transa, int transb, int M, int N, int K, double alpha,
                        const double *A, int lda, const double *B, int ldb, double beta,
                        double *C, int ldc, int block_dim);
void oracle_sgemm_tiled(int transa, int transb, int M, int N, int K, float alpha,
                        const float *A, int lda, const float *B, int ldb, float beta,
                        float *C, int ldc, int block_dim);
/* complex128 interleaved (re, im); alpha/beta point to 2 doubles */
void oracle_zgemm_tiled(int transa, int transb, int M, int N, int K, const double *alpha,
                        const double *A, int lda, const double *B, int ldb, const double *beta,
                        double *C, int ldc, int block_dim);

/* complex64 interleaved (re, im) floats; alpha/beta point to 2 floats */
void oracle_cgemm_tiled(int transa, int transb, int M, int N, int K, const float *alpha,
                        const float *A, int lda, const float *B, int ldb, const float *beta,
                        float *C, int ldc, int block_dim);

/* Sampled entries (ii[t], jj[t]) of alpha*op(A)*op(B) + beta*C0 in double-double.
 * hi/lo: the value as an unevaluated sum; bound: |alpha| sum|a||b| + |beta||c0|.
 * For zgemm hi/lo/bound hold 2 doubles (re, im) per entry; the bound is the
 * same scale for both parts. Pass C0 = NULL when beta is zero. */
void oracle_dgemm_dd_entries(int transa, int transb, int M, int N, int K, double alpha,
                             const double *A, int lda, const double *B, int ldb, double beta,
                             const double *C0, int ldc, int64_t n, const int64_t *ii,
                             const int64_t *jj, double *hi, double *lo, double *bound);
void oracle_sgemm_dd_entries(int transa, int transb, int M, int N, int K, float alpha,
                             const float *A, int lda, const float *B, int ldb, float beta,
                             const float *C0, int ldc, int64_t n, const int64_t *ii,
                             const int64_t *jj, double *hi, double *lo, double *bound);
void oracle_zgemm_dd_entries(int transa, int transb, int M, int N, int K, const double *alpha,
                             const double *A, int lda, const double *B, int ldb,
                             const double *beta, const double *C0, int ldc, int64_t n,
                             const int64_t *ii, const int64_t *jj, double *hi, double *lo,
                             double *bound);

/* OpenBLAS through dlopen. `paths` is a ':'-separated candidate list; each
 * entry is "path|symbol_prefix|ilp64" (ilp64 = 0 or 1). Returns 0 on success. */
int oracle_openblas_open(const char *paths);
const char *oracle_openblas_name(void);
int oracle_openblas_dgemm(int order, int transa, int transb, int M, int N, int K, double alpha,
                          const double *A, int lda, const double *B, int ldb, double beta,
                          double *C, int ldc);
int oracle_openblas_sgemm(int order, int transa, int transb, int M, int N, int K, float alpha,
                          const float *A, int lda, const float *B, int ldb, float beta,
                          float *C, int ldc);
int oracle_openblas_cgemm(int order, int transa, int transb, int M, int N, int K,
                          const float *alpha, const float *A, int lda, const float *B,
                          int ldb, const float *beta, float *C, int ldc);
int oracle_openblas_zgemm(int order, int transa, int transb, int M, int N, int K,
                          const double *alpha, const double *A, int lda, const double *B,
                          int ldb, const double *beta, double *C, int ldc);

/* Seeded generators (SplitMix64 counter RNG) used by tests and bench for
 * reproducible column-major inputs: x[t] = lo + (hi-lo)*u(seed, t). */
void oracle_fill_uniform_f64(double *x, int64_t n, uint64_t seed, double lo, double hi);
void oracle_fill_uniform_f32(float *x, int64_t n, uint64_t seed, float lo, float hi);
/* x[t] = U[-0.5,0.5] * exp(phi * g), g ~ N(0,1) (Box-Muller). */
void oracle_fill_spread_f64(double *x, int64_t n, uint64_t seed, double phi);

#ifdef __cplusplus
}
#endif
#endif
