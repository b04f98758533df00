/*
 * blasx_b200.h -- C ABI of the B200-native GEMM runtime.
 *
 * The first block is the drop-in boundary: the CBLAS and Fortran-77 GEMM
 * symbols of linnanwang/BLASX, with the same signatures, enum values, argument
 * meaning and xerbla_ error reporting. Operands are host-resident and
 * column-major (row-major is accepted too, see below); the call is
 * synchronous: C is complete when it returns.
 *
 * Differences from the reference, on purpose:
 *   - every call with M, N > 0 runs on the GPU (no CPU BLAS, no size
 *     threshold; the reference sends calls with all dims <= 1000 to a CPU
 *     BLAS, blas/dgemm.c:61-64);
 *   - CblasRowMajor is honoured (the reference ignores Order on its GPU path,
 *     blas/dgemm.c:107), using the identity C^T = op(B)^T op(A)^T;
 *   - the calls are thread-safe and re-entrant;
 *   - internal CUDA failures never abort the process: the call reports to
 *     stderr and records the status for blasx_last_status().
 */
#ifndef BLASX_B200_H
#define BLASX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Enum values of the reference's include/cblas.h:11-15 (skipped when a
 * cblas.h guarded by CBLAS_H was included first). */
#if !defined(CBLAS_H) && !defined(CBLAS_ENUM_DEFINED_H)
#define CBLAS_ENUM_DEFINED_H
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
#endif

/* ------------------------------------------------------------------------ */
/* Drop-in boundary                                                          */
/* ------------------------------------------------------------------------ */

/* Replaces cblas_sgemm, include/cblas.h:424 (implementation blas/sgemm.c:16). */
void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const float alpha, const float *A, const int lda, const float *B,
                 const int ldb, const float beta, float *C, const int ldc);

/* Replaces cblas_dgemm, include/cblas.h:454 (implementation blas/dgemm.c:18-128). */
void cblas_dgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const double alpha, const double *A, const int lda, const double *B,
                 const int ldb, const double beta, double *C, const int ldc);

/* Replaces cblas_zgemm, include/cblas.h:514 (implementation blas/zgemm.c:16-130).
 * alpha, beta, A, B, C point to interleaved (re, im) double pairs. */
void cblas_zgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const void *alpha, const void *A, const int lda, const void *B,
                 const int ldb, const void *beta, void *C, const int ldc);

/* Replaces cblas_cgemm, include/cblas.h:484 (implementation blas/cgemm.c:14-106,
 * whose GPU path is commented out: the reference runs every CGEMM on its CPU
 * BLAS). alpha, beta, A, B, C point to interleaved (re, im) float pairs. */
void cblas_cgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const void *alpha, const void *A, const int lda, const void *B,
                 const int ldb, const void *beta, void *C, const int ldc);

/* Replace the F77 wrappers sgemm_ (blas/sgemm.c), dgemm_ (blas/dgemm.c:131-154),
 * cgemm_ (blas/cgemm.c:109-) and zgemm_ (blas/zgemm.c:133-156): every argument
 * by pointer, trans chars 'N'/'T'/'C' in either case, column-major. */
void sgemm_(char *transa, char *transb, int *m, int *n, int *k, float *alpha, float *A,
            int *lda, float *B, int *ldb, float *beta, float *C, int *ldc);
void dgemm_(char *transa, char *transb, int *m, int *n, int *k, double *alpha, double *A,
            int *lda, double *B, int *ldb, double *beta, double *C, int *ldc);
void cgemm_(char *transa, char *transb, int *m, int *n, int *k, float *alpha, float *A,
            int *lda, float *B, int *ldb, float *beta, float *C, int *ldc);
void zgemm_(char *transa, char *transb, int *m, int *n, int *k, double *alpha, double *A,
            int *lda, double *B, int *ldb, double *beta, double *C, int *ldc);

/* Replace cblas_ssyrk / cblas_dsyrk / cblas_zsyrk (include/cblas.h:434,464,524;
 * implementations blas/ssyrk.c, blas/dsyrk.c:15-77, blas/zsyrk.c, which always
 * run on the host BLAS): C = alpha op(A) op(A)^T + beta C on the uplo
 * triangle only, on the GPU. ConjTrans is Trans for the real routines and
 * illegal (info 2) for ZSYRK. */
void cblas_ssyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const float alpha,
                 const float *A, const int lda, const float beta, float *C, const int ldc);
void cblas_dsyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                 const double *A, const int lda, const double beta, double *C, const int ldc);
void cblas_zsyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                 const void *A, const int lda, const void *beta, void *C, const int ldc);

/* Replace cblas_ssyr2k / cblas_dsyr2k / cblas_zsyr2k (include/cblas.h:468;
 * implementations blas/dsyr2k.c:16-86 and siblings, host BLAS only):
 * C = alpha op(A) op(B)^T + alpha op(B) op(A)^T + beta C on the uplo triangle. */
void cblas_ssyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const float alpha,
                  const float *A, const int lda, const float *B, const int ldb, const float beta,
                  float *C, const int ldc);
void cblas_dsyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                  const double *A, const int lda, const double *B, const int ldb, const double beta,
                  double *C, const int ldc);
void cblas_zsyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const void *beta,
                  void *C, const int ldc);

/* Replace cblas_csyrk / cblas_csyr2k (include/cblas.h:494,498; blas/csyrk.c,
 * blas/csyr2k.c, host BLAS only): the complex64 forms of the above (alpha,
 * beta, A, B, C interleaved (re, im) float pairs; ConjTrans illegal). */
void cblas_csyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                 const void *A, const int lda, const void *beta, void *C, const int ldc);
void cblas_csyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const void *beta,
                  void *C, const int ldc);

/* Replace cblas_cherk / cblas_zherk (include/cblas.h:553,568; blas/zherk.c:
 * 14-78, host BLAS only): C = alpha op(A) op(A)^H + beta C on the uplo
 * triangle, alpha and beta real, Trans CblasNoTrans or CblasConjTrans
 * (CblasTrans is illegal, info 2); the imaginary parts of C's diagonal are
 * set to zero. cblas_cher2k / cblas_zher2k (include/cblas.h:557,572;
 * blas/zher2k.c:15-86): C = alpha op(A) op(B)^H + conj(alpha) op(B) op(A)^H
 * + beta C, beta real. ZHER2K reports argument errors under the name
 * "ZHERK", as the reference does (blas/zher2k.c:13). */
void cblas_cherk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const float alpha,
                 const void *A, const int lda, const float beta, void *C, const int ldc);
void cblas_zherk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                 const void *A, const int lda, const double beta, void *C, const int ldc);
void cblas_cher2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const float beta,
                  void *C, const int ldc);
void cblas_zher2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const double beta,
                  void *C, const int ldc);

/* Replace the F77 wrappers ssyrk_ / dsyrk_ (blas/dsyrk.c:80-101) / zsyrk_ and
 * ssyr2k_ / dsyr2k_ (blas/dsyr2k.c:88-) / zsyr2k_: uplo 'U'/'L', trans
 * 'N'/'T'/'C', column-major, every argument by pointer. */
void ssyrk_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda,
            float *beta, float *C, int *ldc);
void dsyrk_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
            double *beta, double *C, int *ldc);
void zsyrk_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
            double *beta, double *C, int *ldc);
void ssyr2k_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *B,
             int *ldb, float *beta, float *C, int *ldc);
void dsyr2k_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
             double *B, int *ldb, double *beta, double *C, int *ldc);
void zsyr2k_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
             double *B, int *ldb, double *beta, double *C, int *ldc);
/* csyrk_ / csyr2k_ (complex64 scalars as (re, im) float pairs), cherk_ /
 * zherk_ (real alpha, beta) and cher2k_ / zher2k_ (complex alpha, real beta):
 * blas/csyrk.c:76-, blas/zherk.c:81-104, blas/zher2k.c:89-118. */
void csyrk_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *beta,
            float *C, int *ldc);
void csyr2k_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *B,
             int *ldb, float *beta, float *C, int *ldc);
void cherk_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *beta,
            float *C, int *ldc);
void zherk_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda, double *beta,
            double *C, int *ldc);
void cher2k_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *B, int *ldb,
             float *beta, float *C, int *ldc);
void zher2k_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda, double *B,
             int *ldb, double *beta, double *C, int *ldc);

/* Replace cblas_ssymm / cblas_dsymm / cblas_csymm / cblas_zsymm
 * (include/cblas.h:429,459,489,519; implementations blas/dsymm.c:16-72 and
 * siblings, which always run on the host BLAS) and cblas_chemm / cblas_zhemm
 * (include/cblas.h:548,563; blas/zhemm.c:16-77): C = alpha A B + beta C (Side
 * Left, A M x M) or alpha B A + beta C (Right, A N x N), A symmetric
 * (Hermitian for ?hemm) and read from its Uplo triangle only. On the GPU:
 * the stored triangle is completed on the device, then the GEMM runs. */
void cblas_ssymm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const int M, const int N, const float alpha,
                 const float *A, const int lda, const float *B, const int ldb, const float beta,
                 float *C, const int ldc);
void cblas_dsymm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const int M, const int N, const double alpha,
                 const double *A, const int lda, const double *B, const int ldb, const double beta,
                 double *C, const int ldc);
void cblas_csymm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const int M, const int N, const void *alpha,
                 const void *A, const int lda, const void *B, const int ldb, const void *beta,
                 void *C, const int ldc);
void cblas_zsymm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const int M, const int N, const void *alpha,
                 const void *A, const int lda, const void *B, const int ldb, const void *beta,
                 void *C, const int ldc);
void cblas_chemm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const int M, const int N, const void *alpha,
                 const void *A, const int lda, const void *B, const int ldb, const void *beta,
                 void *C, const int ldc);
void cblas_zhemm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const int M, const int N, const void *alpha,
                 const void *A, const int lda, const void *B, const int ldb, const void *beta,
                 void *C, const int ldc);

/* Replace cblas_strmm / cblas_dtrmm / cblas_ctrmm / cblas_ztrmm
 * (include/cblas.h:443,473,503,533; implementations blas/dtrmm.c:17-64 and
 * siblings, host BLAS only): B = alpha op(A) B (Side Left) or alpha B op(A)
 * (Right), A triangular (Uplo, Diag), op(A) = A, A^T or A^H. B is read whole
 * before the product overwrites it. */
void cblas_strmm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const float alpha,
                 const float *A, const int lda, float *B, const int ldb);
void cblas_dtrmm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb);
void cblas_ctrmm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const void *alpha,
                 const void *A, const int lda, void *B, const int ldb);
void cblas_ztrmm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const void *alpha,
                 const void *A, const int lda, void *B, const int ldb);

/* Replace cblas_strsm / cblas_dtrsm / cblas_ctrsm / cblas_ztrsm
 * (include/cblas.h:448,478,508,538; implementations blas/dtrsm.c:16-75 and
 * siblings, host BLAS only): solves op(A) X = alpha B (Side Left) or
 * X op(A) = alpha B (Right) for X, which overwrites B; A triangular (Uplo,
 * Diag), op(A) = A, A^T or A^H. Only the Uplo triangle of A is read, and not
 * its diagonal when Diag is CblasUnit. */
void cblas_strsm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const float alpha,
                 const float *A, const int lda, float *B, const int ldb);
void cblas_dtrsm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const double alpha,
                 const double *A, const int lda, double *B, const int ldb);
void cblas_ctrsm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const void *alpha,
                 const void *A, const int lda, void *B, const int ldb);
void cblas_ztrsm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,
                 const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_DIAG Diag, const int M, const int N, const void *alpha,
                 const void *A, const int lda, void *B, const int ldb);

/* Replace the F77 wrappers ?symm_ (blas/dsymm.c:74-95), ?hemm_ (blas/zhemm.c:
 * 80-99), ?trmm_ (blas/dtrmm.c:67-91) and ?trsm_ (blas/dtrsm.c:78-100): side
 * 'L'/'R', uplo 'U'/'L', transa 'N'/'T'/'C', diag 'N'/'U', column-major, every
 * argument by pointer; complex scalars are (re, im) pairs. */
void ssymm_(char *side, char *uplo, int *m, int *n, float *alpha, float *A, int *lda, float *B,
            int *ldb, float *beta, float *C, int *ldc);
void dsymm_(char *side, char *uplo, int *m, int *n, double *alpha, double *A, int *lda, double *B,
            int *ldb, double *beta, double *C, int *ldc);
void csymm_(char *side, char *uplo, int *m, int *n, float *alpha, float *A, int *lda, float *B,
            int *ldb, float *beta, float *C, int *ldc);
void zsymm_(char *side, char *uplo, int *m, int *n, double *alpha, double *A, int *lda, double *B,
            int *ldb, double *beta, double *C, int *ldc);
void chemm_(char *side, char *uplo, int *m, int *n, float *alpha, float *A, int *lda, float *B,
            int *ldb, float *beta, float *C, int *ldc);
void zhemm_(char *side, char *uplo, int *m, int *n, double *alpha, double *A, int *lda, double *B,
            int *ldb, double *beta, double *C, int *ldc);
void strmm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, float *alpha,
            float *A, int *lda, float *B, int *ldb);
void dtrmm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, double *alpha,
            double *A, int *lda, double *B, int *ldb);
void ctrmm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, float *alpha,
            float *A, int *lda, float *B, int *ldb);
void ztrmm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, double *alpha,
            double *A, int *lda, double *B, int *ldb);
void strsm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, float *alpha,
            float *A, int *lda, float *B, int *ldb);
void dtrsm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, double *alpha,
            double *A, int *lda, double *B, int *ldb);
void ctrsm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, float *alpha,
            float *A, int *lda, float *B, int *ldb);
void ztrsm_(char *side, char *uplo, char *transa, char *diag, int *m, int *n, double *alpha,
            double *A, int *lda, double *B, int *ldb);

/* Replaces xerbla_, blas/error.c:5: prints
 * " ** On entry to <NAME> parameter number <info> had an illegal value".
 * Exported weak, so an application's own xerbla_ takes precedence. */
void xerbla_(char *name, int *info);

/* ------------------------------------------------------------------------ */
/* Extensions (no counterpart in the reference)                              */
/* ------------------------------------------------------------------------ */

/* Status codes returned by the blasx_* calls and recorded per thread. */
enum blasx_status {
    BLASX_OK = 0,
    BLASX_ERR_ARG = 1,      /* illegal argument (xerbla_ was called) */
    BLASX_ERR_CUDA = 2,     /* a CUDA runtime call failed */
    BLASX_ERR_NOMEM = 3,    /* device allocation or budget exhausted */
    BLASX_ERR_NODEVICE = 4, /* no usable GPU */
    BLASX_ERR_TIMEOUT = 5,  /* a bounded device wait ran out */
    BLASX_ERR_UNSUPPORTED = 6,
    BLASX_ERR_CLOSED = 7    /* the serving loop was shut down */
};

/* Status of the calling thread's last GEMM call and its message. */
int blasx_last_status(void);
const char *blasx_last_error(void);

/* DGEMM/ZGEMM precision mode: 0 = auto (Ozaki emulation when the measured
 * exponent spread allows FP64 accuracy, native FP64 otherwise),
 * 1 = native FP64 only, 2 = Ozaki emulation whenever it is feasible.
 * Also read once from the environment variable BLASX_DGEMM_MODE
 * (auto|native|ozaki). Returns the previous mode. */
int blasx_set_dgemm_mode(int mode);

/* Device tile-cache byte budget (0 = default: 90% of free HBM at first use;
 * env BLASX_HBM_BUDGET, bytes, suffixes K/M/G accepted). Takes effect for
 * calls that start after it returns. Returns 0 on success. */
int blasx_set_hbm_budget(size_t bytes);

/* Tile edge (rows = cols) used by the host pipeline, 0 = automatic
 * (env BLASX_TILE). Multiple of 256, between 256 and 16384. */
int blasx_set_tile(int tile);

/* Pageable host memory passed to a host call (memory that is neither
 * pinned nor device memory): 1 = staged through a ring of pinned bounce
 * buffers, packed and unpacked by host threads while the copy engines run
 * (default); 0 = registered for the duration of the call (cudaHostRegister,
 * as the reference does in blas/dgemm.c:88-121). Also read once from the
 * environment variable BLASX_HOST_STAGING (0/off). Returns the previous
 * setting. */
int blasx_set_host_staging(int on);

/* Per-call statistics of the calling thread's last host GEMM call. */
typedef struct blasx_call_stats {
    double seconds;           /* wall time of the call */
    double h2d_bytes;         /* bytes copied host -> device */
    double d2h_bytes;         /* bytes copied device -> host */
    double cache_hits;        /* operand tiles found resident */
    double cache_misses;      /* operand tiles copied in */
    double evictions;         /* operand tiles evicted */
    int path;                 /* 1 native, 2 Ozaki emulation, 3 scale-only,
                                 4 emulation requested, native chosen on the
                                 device (spread too wide or non-finite input) */
    int moduli;               /* Ozaki moduli used (0 when native) */
    int tile;                 /* tile edge used */
    int host_copy;            /* host memory: 0 copied directly (pinned by
                                 the caller), 1 staged through bounce buffers,
                                 2 registered for the call */
} blasx_call_stats;
void blasx_get_call_stats(blasx_call_stats *out);

/* Tile schedule of a host GEMM that does not fit the HBM budget, computed on
 * the host without touching a GPU (no counterpart in the reference; it
 * replaces the reference's task queue and LRU tile cache,
 * blas/blasx_task_queue.c, blas/LRU.c). C is cut into tile x tile blocks
 * visited in bands of two block rows, column by column, snaking (row by row
 * when that loads fewer tiles); operand tiles occupy budget_bytes / (tile^2 *
 * elem_bytes) - 3 slots (3 hold C tiles); policy 0 = Belady (farthest next
 * use), 1 = LRU. */
typedef struct blasx_tile_plan_stats {
    int tiles_m, tiles_n, tiles_k, slots;
    long long steps;           /* GEMM launches (C tiles x K-steps) */
    long long tile_loads;      /* operand tiles copied host -> device */
    long long tile_hits;       /* operand uses served from HBM */
    long long evictions;
    double operand_h2d_bytes;  /* bytes of A and B tiles copied in */
    double min_operand_h2d_bytes;  /* each element of A and B copied once */
} blasx_tile_plan_stats;
int blasx_tile_plan(long long M, long long N, long long K, long long tile,
                    long long budget_bytes, int elem_bytes, int policy,
                    blasx_tile_plan_stats *out);

/* Device-resident GEMM: A, B, C are device pointers (column-major), the call
 * is enqueued on `stream` (a cudaStream_t; NULL = the CUDA default stream)
 * and returns without waiting. Scalars are host values. Used by callers whose
 * operands already live in HBM. Returns a blasx_status. */
int blasx_dgemm_device(int transa, int transb, int M, int N, int K, double alpha,
                       const double *A, int lda, const double *B, int ldb, double beta,
                       double *C, int ldc, void *stream);

int blasx_sgemm_device(int transa, int transb, int M, int N, int K, float alpha,
                       const float *A, int lda, const float *B, int ldb, float beta, float *C,
                       int ldc, void *stream);
int blasx_zgemm_device(int transa, int transb, int M, int N, int K, const void *alpha,
                       const void *A, int lda, const void *B, int ldb, const void *beta,
                       void *C, int ldc, void *stream);
/* complex64: alpha, beta, A, B, C are interleaved (re, im) float pairs. */
int blasx_cgemm_device(int transa, int transb, int M, int N, int K, const void *alpha,
                       const void *A, int lda, const void *B, int ldb, const void *beta,
                       void *C, int ldc, void *stream);

/* Device-resident DSYRK (column-major, uplo CblasUpper/CblasLower, trans
 * CblasNoTrans/CblasTrans): C = alpha op(A) op(A)^T + beta C on the uplo
 * triangle of the device matrix C, enqueued on `stream`; returns a status.
 * No counterpart in the reference. */
int blasx_dsyrk_device(int uplo, int trans, int N, int K, double alpha, const double *A, int lda,
                       double beta, double *C, int ldc, void *stream);

/* Device-resident DTRSM (column-major; side CblasLeft/CblasRight, uplo, trans,
 * diag as for cblas_dtrsm): solves op(A) X = alpha B or X op(A) = alpha B for
 * the device matrix B (overwritten by X), enqueued on `stream`; returns a
 * status. Update GEMMs follow the precision mode. No counterpart in the
 * reference. */
int blasx_dtrsm_device(int side, int uplo, int trans, int diag, int M, int N, double alpha,
                       const double *A, int lda, double *B, int ldb, void *stream);

/* Device-resident DTRMM (arguments as for cblas_dtrmm, column-major): B =
 * alpha op(A) B or alpha B op(A) on the device matrix B, in place, enqueued on
 * `stream`; returns a status. Its small leaf scratch is allocated and freed
 * stream-ordered on `stream`. No counterpart in the reference. */
int blasx_dtrmm_device(int side, int uplo, int trans, int diag, int M, int N, double alpha,
                       const double *A, int lda, double *B, int ldb, void *stream);

/* Device-resident DGEMM that allocates no memory. No counterpart in the
 * reference. It is meant for callers that cannot let a library call
 * cudaMalloc: a framework whose own allocator has already reserved the
 * GPU's memory (a cudaMalloc would fail or fragment that pool), or
 * latency-critical code where cudaMalloc / cudaFree may synchronise the
 * device. Arguments as for blasx_dgemm_device; the caller still provides A,
 * B and C. The precision mode (blasx_set_dgemm_mode) applies: in native mode
 * the FP64 kernel runs; in auto mode the emulated (INT8 Ozaki) path runs,
 * with the native FP64 kernel chosen on the device when the operands' spread
 * is too wide (unlike blasx_dgemm_device, auto mode does not send small
 * problems to the native kernel by size); in ozaki mode the emulated path
 * always runs. Its scratch is a fixed 64 MiB device array that every GPU
 * loading this library holds until the process exits; emulated problems
 * whose scratch would not fit (M = N = K = 1024 fits; 2048 does not) are
 * rejected with BLASX_ERR_UNSUPPORTED and a message in blasx_last_error().
 * The first call on each device context performs a one-time set-up there
 * (it looks up the array's device address and uploads constant tables);
 * make that first call before any stream capture. All calls share the one
 * array: calls that overlap on the GPU (other streams, other threads) race
 * and must be serialised by the caller. Returns a blasx_status for what
 * the host could check; a failure on the device is reported by
 * blasx_dgemm_device_noalloc_status. */
int blasx_dgemm_device_noalloc(int transa, int transb, int M, int N, int K, double alpha,
                               const double *A, int lda, const double *B, int ldb,
                               double beta, double *C, int ldc, void *stream);

/* Device status of the last blasx_dgemm_device_noalloc call on the current
 * device: waits for `stream` (the stream that call was enqueued on), then
 * reads the shared scratch's error word. Returns BLASX_ERR_TIMEOUT when a
 * bounded wait of the residue GEMM ran out in that call (its C is then
 * undefined), else BLASX_OK. Allocates nothing. No counterpart in the
 * reference. */
int blasx_dgemm_device_noalloc_status(void *stream);

/* Number of kernels this library has launched since it was loaded (all
 * threads); lets a caller count the GPU work of a region. */
uint64_t blasx_kernel_launch_count(void);

/* Test hooks (no counterpart in the reference, which assert()s on every CUDA
 * failure, blas/LRU.c:118,134). They drive the error paths without faulting
 * the GPU.
 *
 * blasx_test_stall_residue_gemm: the next `launches` launches of the INT8
 * residue GEMM run with every mbarrier wait limited to `wait_cycles` clock
 * cycles (default about one second), and their CTA 0 issues no loads for
 * its second pipeline stage, so the MMA issuer's wait for that stage runs
 * out: the kernel raises its device error word, waits for its own copies and
 * MMAs, frees its tensor memory and returns. The call that launched it
 * reports BLASX_ERR_TIMEOUT; its C is undefined.
 *
 * blasx_test_fail_allocation: the nth device allocation of the library from
 * now on (1 = the next one) reports an out-of-memory error without
 * allocating; 0 disarms. */
int blasx_test_stall_residue_gemm(int launches, long long wait_cycles);
int blasx_test_fail_allocation(int nth);

/* Serving loop (no counterpart in the reference, whose GEMM path is not
 * re-entrant). While it runs, cblas_?gemm / ?gemm_ calls from any number of
 * host threads are queued to one scheduler thread that owns the device: it
 * admits requests when an in-flight slot is free and their device memory
 * fits hbm_budget (0 = 85% of free HBM), copies each one's operands on its
 * own stream, and runs the compute of every request in flight in one
 * persistent kernel whose CTAs take the tiles of all of them from a task
 * queue the scheduler fills (continuous batching: native FP64 / complex128 /
 * FP32 / complex64 tiles and every stage of emulated requests mix on the
 * SMs); it keeps copies of B operands in an HBM operand cache of cache_bytes
 * (0 = a quarter of the budget).
 * Operand identity: host pointer, leading dimension, stored shape, dtype and
 * a fingerprint of 1024 sampled elements plus the first and last column; a
 * caller that modifies an operand in place without touching those must call
 * blasx_serve_invalidate(ptr). max_inflight: requests on the device at once
 * (0 = 8, at most 64). Calls block until their C is complete. */
int blasx_serve_start(size_t hbm_budget, size_t cache_bytes, int max_inflight);
/* Drains queued and in-flight requests, then stops; call once no thread is
 * still submitting. */
int blasx_serve_stop(void);
/* Drops cached device copies of the operand at host_ptr; returns how many. */
int blasx_serve_invalidate(const void *host_ptr);
typedef struct blasx_serve_stats {
    long long submitted, completed, failed;
    long long cache_hits, cache_misses;        /* B operands reused / copied */
    long long grouped_launches, grouped_requests; /* persistent-kernel launches; requests run by it */
    int max_inflight_seen, reserved;
    double p50_ms, p99_ms, mean_ms, max_ms;    /* submit -> completion */
    double flops, seconds, tflops;             /* first submit -> last completion */
    double admit_seconds, admit_max_ms;        /* scheduler time spent enqueueing requests */
    long long memory_waits;                    /* admission passes over a request that did not fit */
    long long head_holds;                      /* passes stopped to keep memory for the oldest request */
    double alloc_seconds, copy_seconds;        /* parts of admit_seconds: device allocation, copy calls */
    double compute_enqueue_seconds;            /* part of admit_seconds: enqueueing the GEMM kernels */
    double mean_copy_in_ms, mean_compute_ms, mean_copy_out_ms; /* per request: admitted -> operands on the
                                                  device -> result computed -> result on the host */
} blasx_serve_stats;
void blasx_serve_get_stats(blasx_serve_stats *out);
int blasx_serve_reset_stats(void);

/* Per-phase device timing. When enabled, every GEMM records CUDA events on
 * its own stream around its phases: 0 slicing (emulated path: statistics,
 * modulus decision, scaling, residues), 1 INT8 residue GEMMs, 2 CRT
 * reconstruction and epilogue, 3 native kernel. blasx_profile_enable resets
 * the totals and returns the previous setting; blasx_profile_read waits for
 * the recorded events, writes up to n totals (milliseconds) and span counts,
 * and returns the number of phases. */
int blasx_profile_enable(int on);
int blasx_profile_read(double *ms, long *count, int n);

/* Release all device memory and streams held by the library (the next call
 * re-initialises). Returns a blasx_status. */
int blasx_finalize(void);

#ifdef __cplusplus
}
#endif
#endif /* BLASX_B200_H */
