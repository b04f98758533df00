// gemm_api.cu -- the drop-in C ABI: cblas_?gemm, ?gemm_, xerbla_, and the
// device-resident blasx_?gemm_device extensions.
//
// Argument checking follows the reference exactly for column-major calls
// (blas/dgemm.c:28-57, blas/sgemm.c, blas/zgemm.c:24-56): info 1 TransA,
// 2 TransB, 3 M, 4 N, 5 K, 8 lda, 10 ldb, 13 ldc, reported through xerbla_
// with C untouched. The F77 wrappers keep the reference's numbering, where a
// bad TransB overrides a bad TransA (blas/dgemm.c:140-146).
#include <cstdio>

#include "host_pipeline.h"
#include "kernels.h"
#include "runtime.h"
#include "serving.h"

extern "C" __attribute__((weak)) void xerbla_(char *name, int *info) {
    // Same text as the reference, blas/error.c:5-8.
    printf(" ** On entry to %6s parameter number %2d had an illegal value\n", name, *info);
}

namespace bx {
namespace {

bool trans_ok(int t) { return t == NoTrans || t == TransT || t == ConjT; }

// Returns the reference's info code (0 = arguments legal). Row-major calls
// are checked with row-major leading-dimension rules.
int check_args(int order, int ta, int tb, int M, int N, int K, int lda, int ldb, int ldc) {
    const bool row = (order == CblasRowMajor);
    int nrowa, nrowb;
    if (!row) {
        nrowa = (ta == NoTrans) ? M : K;
        nrowb = (tb == NoTrans) ? K : N;
    } else {
        nrowa = (ta == NoTrans) ? K : M;
        nrowb = (tb == NoTrans) ? N : K;
    }
    const int nrowc = row ? N : M;
    auto mx1 = [](int v) { return v > 1 ? v : 1; };
    if (!trans_ok(ta)) return 1;
    if (!trans_ok(tb)) return 2;
    if (M < 0) return 3;
    if (N < 0) return 4;
    if (K < 0) return 5;
    if (lda < mx1(nrowa)) return 8;
    if (ldb < mx1(nrowb)) return 10;
    if (ldc < mx1(nrowc)) return 13;
    return 0;
}

// Builds the column-major problem. Row-major C = op(A) op(B) is the
// column-major C^T = op(B)^T op(A)^T: swap the operands and M/N.
Gemm make_gemm(DType dt, int order, int ta, int tb, int M, int N, int K, cplx alpha,
               const void *A, int lda, const void *B, int ldb, cplx beta, void *C, int ldc) {
    Gemm g;
    g.dt = dt;
    if (!is_complex(dt)) {  // ConjTrans on real data is Trans
        if (ta == ConjT) ta = TransT;
        if (tb == ConjT) tb = TransT;
    }
    if (order == CblasRowMajor) {
        g.ta = tb; g.tb = ta;
        g.M = N; g.N = M; g.K = K;
        g.A = B; g.lda = ldb; g.B = A; g.ldb = lda;
    } else {
        g.ta = ta; g.tb = tb;
        g.M = M; g.N = N; g.K = K;
        g.A = A; g.lda = lda; g.B = B; g.ldb = ldb;
    }
    g.alpha = alpha; g.beta = beta;
    g.C = C; g.ldc = ldc;
    return g;
}

void host_entry(const char *name, DType dt, int order, int ta, int tb, int M, int N, int K,
                cplx alpha, const void *A, int lda, const void *B, int ldb, cplx beta, void *C,
                int ldc) {
    clear_error();
    int info = check_args(order, ta, tb, M, N, K, lda, ldb, ldc);
    if (info) {
        set_error(BLASX_ERR_ARG, "%s parameter %d illegal", name, info);
        xerbla_(const_cast<char *>(name), &info);
        return;
    }
    Gemm g = make_gemm(dt, order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    if (g.M == 0 || g.N == 0) return;  // quick return, as in BLAS
    if (serve::active()) serve::submit(g);  // records its own status
    else host_gemm(g);
}

int device_entry(DType dt, int ta, int tb, int M, int N, int K, cplx alpha, const void *A,
                 int lda, const void *B, int ldb, cplx beta, void *C, int ldc, void *stream) {
    clear_error();
    int info = check_args(CblasColMajor, ta, tb, M, N, K, lda, ldb, ldc);
    if (info) return set_error(BLASX_ERR_ARG, "device gemm parameter %d illegal", info);
    Gemm g = make_gemm(dt, CblasColMajor, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    Context *c = context();
    if (!c) return last_status();
    // NULL is the CUDA legacy default stream, as everywhere in the CUDA API
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (g.alpha_zero() || g.K == 0) return launch_scale(g, s);
    return device_gemm(g, s);
}

bool f77_trans(const char *c, int *t) {
    switch (*c) {
        case 'N': case 'n': *t = NoTrans; return true;
        case 'T': case 't': *t = TransT; return true;
        case 'C': case 'c': *t = ConjT; return true;
        default: return false;
    }
}

}  // namespace

int gemm_arg_info(int order, int ta, int tb, int M, int N, int K, int lda, int ldb, int ldc) {
    return check_args(order, ta, tb, M, N, K, lda, ldb, ldc);
}

}  // namespace bx

using bx::cplx;
using bx::DType;

extern "C" {

void cblas_sgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const float alpha, const float *A, const int lda, const float *B,
                 const int ldb, const float beta, float *C, const int ldc) {
    bx::host_entry("SGEMM ", DType::F32, Order, TransA, TransB, M, N, K, cplx{alpha, 0}, A, lda,
                   B, ldb, cplx{beta, 0}, C, ldc);
}

void cblas_dgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const double alpha, const double *A, const int lda, const double *B,
                 const int ldb, const double beta, double *C, const int ldc) {
    bx::host_entry("DGEMM ", DType::F64, Order, TransA, TransB, M, N, K, cplx{alpha, 0}, A, lda,
                   B, ldb, cplx{beta, 0}, C, ldc);
}

void cblas_zgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const void *alpha, const void *A, const int lda, const void *B,
                 const int ldb, const void *beta, void *C, const int ldc) {
    const double *al = static_cast<const double *>(alpha);
    const double *be = static_cast<const double *>(beta);
    bx::host_entry("ZGEMM ", DType::C128, Order, TransA, TransB, M, N, K, cplx{al[0], al[1]}, A,
                   lda, B, ldb, cplx{be[0], be[1]}, C, ldc);
}

// Replaces the reference's cblas_cgemm (blas/cgemm.c:14-106), whose GPU path
// is commented out so that every call runs on its CPU BLAS. alpha, beta, A, B
// and C point to interleaved (re, im) float pairs.
void cblas_cgemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,
                 const enum CBLAS_TRANSPOSE TransB, const int M, const int N, const int K,
                 const void *alpha, const void *A, const int lda, const void *B,
                 const int ldb, const void *beta, void *C, const int ldc) {
    const float *al = static_cast<const float *>(alpha);
    const float *be = static_cast<const float *>(beta);
    bx::host_entry("CGEMM ", DType::C64, Order, TransA, TransB, M, N, K, cplx{al[0], al[1]}, A,
                   lda, B, ldb, cplx{be[0], be[1]}, C, ldc);
}

#define BX_F77_PROLOGUE(NAME)                                   \
    int ta = 0, tb = 0, info = -1;                              \
    if (!bx::f77_trans(transa, &ta)) info = 1;                  \
    if (!bx::f77_trans(transb, &tb)) info = 2;                  \
    if (info >= 0) {                                            \
        bx::set_error(BLASX_ERR_ARG, NAME "parameter %d illegal", info); \
        xerbla_(const_cast<char *>(NAME), &info);               \
        return;                                                 \
    }

void sgemm_(char *transa, char *transb, int *m, int *n, int *k, float *alpha, float *A,
            int *lda, float *B, int *ldb, float *beta, float *C, int *ldc) {
    BX_F77_PROLOGUE("SGEMM ")
    cblas_sgemm(CblasColMajor, CBLAS_TRANSPOSE(ta), CBLAS_TRANSPOSE(tb), *m, *n, *k, *alpha, A,
                *lda, B, *ldb, *beta, C, *ldc);
}

void dgemm_(char *transa, char *transb, int *m, int *n, int *k, double *alpha, double *A,
            int *lda, double *B, int *ldb, double *beta, double *C, int *ldc) {
    BX_F77_PROLOGUE("DGEMM ")
    cblas_dgemm(CblasColMajor, CBLAS_TRANSPOSE(ta), CBLAS_TRANSPOSE(tb), *m, *n, *k, *alpha, A,
                *lda, B, *ldb, *beta, C, *ldc);
}

void cgemm_(char *transa, char *transb, int *m, int *n, int *k, float *alpha, float *A,
            int *lda, float *B, int *ldb, float *beta, float *C, int *ldc) {
    BX_F77_PROLOGUE("CGEMM ")
    cblas_cgemm(CblasColMajor, CBLAS_TRANSPOSE(ta), CBLAS_TRANSPOSE(tb), *m, *n, *k, alpha, A,
                *lda, B, *ldb, beta, C, *ldc);
}

void zgemm_(char *transa, char *transb, int *m, int *n, int *k, double *alpha, double *A,
            int *lda, double *B, int *ldb, double *beta, double *C, int *ldc) {
    BX_F77_PROLOGUE("ZGEMM ")
    cblas_zgemm(CblasColMajor, CBLAS_TRANSPOSE(ta), CBLAS_TRANSPOSE(tb), *m, *n, *k, alpha, A,
                *lda, B, *ldb, beta, C, *ldc);
}

int blasx_dgemm_device(int transa, int transb, int M, int N, int K, double alpha,
                       const double *A, int lda, const double *B, int ldb, double beta,
                       double *C, int ldc, void *stream) {
    return bx::device_entry(DType::F64, transa, transb, M, N, K, cplx{alpha, 0}, A, lda, B, ldb,
                            cplx{beta, 0}, C, ldc, stream);
}

int blasx_sgemm_device(int transa, int transb, int M, int N, int K, float alpha,
                       const float *A, int lda, const float *B, int ldb, float beta, float *C,
                       int ldc, void *stream) {
    return bx::device_entry(DType::F32, transa, transb, M, N, K, cplx{alpha, 0}, A, lda, B, ldb,
                            cplx{beta, 0}, C, ldc, stream);
}

int blasx_zgemm_device(int transa, int transb, int M, int N, int K, const void *alpha,
                       const void *A, int lda, const void *B, int ldb, const void *beta,
                       void *C, int ldc, void *stream) {
    const double *al = static_cast<const double *>(alpha);
    const double *be = static_cast<const double *>(beta);
    return bx::device_entry(DType::C128, transa, transb, M, N, K, cplx{al[0], al[1]}, A, lda, B,
                            ldb, cplx{be[0], be[1]}, C, ldc, stream);
}

int blasx_cgemm_device(int transa, int transb, int M, int N, int K, const void *alpha,
                       const void *A, int lda, const void *B, int ldb, const void *beta,
                       void *C, int ldc, void *stream) {
    const float *al = static_cast<const float *>(alpha);
    const float *be = static_cast<const float *>(beta);
    return bx::device_entry(DType::C64, transa, transb, M, N, K, cplx{al[0], al[1]}, A, lda, B,
                            ldb, cplx{be[0], be[1]}, C, ldc, stream);
}

}  // extern "C"
