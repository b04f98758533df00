// syrk_api.cu -- cblas_?syrk / ?syrk_ and cblas_?syr2k / ?syr2k_ (S/D/C/Z), and
// cblas_?herk / ?herk_ and cblas_?her2k / ?her2k_ (C/Z), on the GPU.
//
// The reference declares these (include/cblas.h:434,464,468,524) but always
// runs them on the host BLAS (blas/dsyrk.c:36-39 sets the dispatch type to the
// CPU in every branch; blas/dsyr2k.c likewise). Here they run on the GEMM
// machinery with a triangular output:
//   SYRK   C = alpha op(A) op(A)^T + beta C, only the uplo triangle of C is
//          read or written. op(A) = A (N x K) for Trans = N, A^T for T. It is
//          the GEMM op(A) x op(A)^T on one buffer: the emulated path slices A
//          once and uses the same slices for both operands (real types).
//   SYR2K  C = alpha op(A) op(B)^T + alpha op(B) op(A)^T + beta C: two
//          triangular GEMMs, the second accumulating onto the first (beta 1).
//   HERK   C = alpha op(A) op(A)^H + beta C, alpha and beta real, op(A) = A
//          or A^H; HER2K C = alpha op(A) op(B)^H + conj(alpha) op(B) op(A)^H
//          + beta C. The triangular GEMM with a conjugate transpose; the
//          imaginary parts of C's diagonal are set to zero on the device
//          (Gemm::herm_out), as BLAS specifies.
// The precision mode applies as for GEMM (emulated where it pays, native
// otherwise, decided per call on the shape and on the device per data).
//
// Argument checks follow the reference (blas/dsyrk.c:27-37, blas/dsyr2k.c:
// 43-52): info 1 Uplo, 2 Trans, 3 N, 4 K, 7 lda, then 10 ldc (SYRK) or 9 ldb,
// 12 ldc (SYR2K); the lowest-numbered illegal argument is reported through
// xerbla_. Row-major calls use the row-major leading-dimension rule (the
// reference ignores Order). ConjTrans is Trans for the real routines and illegal (2) for
// ZSYRK / ZSYR2K, as in reference BLAS (the reference's own check lets it
// through to its CPU BLAS, which rejects it).
#include "host_pipeline.h"
#include "kernels.h"
#include "runtime.h"
#include "serving.h"

namespace bx {
namespace {

int to_uplo(int u) { return u == CblasUpper ? 1 : (u == CblasLower ? 2 : 0); }

int check_syr(DType dt, int order, int uplo, int trans, int N, int K, int lda, int ldb, int ldc, bool two) {
    const bool trans_ok = trans == NoTrans || trans == TransT || (trans == ConjT && !is_complex(dt));
    // stored rows of A (and B): op(A) is N x K; row-major storage is the transpose
    const bool rows_n = (trans == NoTrans) != (order == CblasRowMajor);
    const int nrowa = rows_n ? N : K;
    auto mx1 = [](int v) { return v > 1 ? v : 1; };
    if (!to_uplo(uplo)) return 1;
    if (!trans_ok) return 2;
    if (N < 0) return 3;
    if (K < 0) return 4;
    if (lda < mx1(nrowa)) return 7;
    if (two && ldb < mx1(nrowa)) return 9;
    if (ldc < mx1(N)) return two ? 12 : 10;
    return 0;
}

// op(X) op(Y)^T as a column-major GEMM with a triangular output. Row-major
// storage is the column-major transpose: the triangle and the transposition
// both flip.
Gemm tri_gemm(DType dt, int order, int uplo, int trans, int N, int K, cplx alpha, const void *X,
              int ldx, const void *Y, int ldy, cplx beta, void *C, int ldc) {
    int u = to_uplo(uplo);
    bool tr = trans != NoTrans;
    if (order == CblasRowMajor) {
        u = 3 - u;
        tr = !tr;
    }
    Gemm g;
    g.dt = dt;
    g.M = N; g.N = N; g.K = K;
    g.ta = tr ? TransT : NoTrans;  // op(X): N x K
    g.tb = tr ? NoTrans : TransT;  // op(Y)^T: K x N, from the same storage as op(X)
    g.A = X; g.lda = ldx;
    g.B = Y; g.ldb = ldy;
    g.alpha = alpha; g.beta = beta;
    g.C = C; g.ldc = ldc;
    g.uplo = u;
    g.diag = 0;
    return g;
}

void run(const Gemm &g) {
    if (serve::active()) serve::submit(g);
    else host_gemm(g);
}

void syrk_entry(const char *name, DType dt, int order, int uplo, int trans, int N, int K, cplx alpha,
                const void *A, int lda, cplx beta, void *C, int ldc) {
    clear_error();
    int info = check_syr(dt, order, uplo, trans, N, K, lda, 0, ldc, false);
    if (info) {
        set_error(BLASX_ERR_ARG, "%s parameter %d illegal", name, info);
        xerbla_(const_cast<char *>(name), &info);
        return;
    }
    if (N == 0) return;
    run(tri_gemm(dt, order, uplo, trans, N, K, alpha, A, lda, A, lda, beta, C, ldc));
}

void syr2k_entry(const char *name, DType dt, int order, int uplo, int trans, int N, int K,
                 cplx alpha, const void *A, int lda, const void *B, int ldb, cplx beta, void *C,
                 int ldc) {
    clear_error();
    int info = check_syr(dt, order, uplo, trans, N, K, lda, ldb, ldc, true);
    if (info) {
        set_error(BLASX_ERR_ARG, "%s parameter %d illegal", name, info);
        xerbla_(const_cast<char *>(name), &info);
        return;
    }
    if (N == 0) return;
    run(tri_gemm(dt, order, uplo, trans, N, K, alpha, A, lda, B, ldb, beta, C, ldc));
    if (last_status() != BLASX_OK) return;
    if (alpha.re == 0 && alpha.im == 0) return;  // the first call already scaled C by beta
    run(tri_gemm(dt, order, uplo, trans, N, K, alpha, B, ldb, A, lda, cplx{1.0, 0.0}, C, ldc));
}

// HERK / HER2K (blas/zherk.c:30-40, blas/zher2k.c:41-47): info 1 Uplo, 2 Trans
// (NoTrans or ConjTrans; Trans is illegal), 3 N, 4 K, 7 lda, then 10 ldc
// (HERK) or 9 ldb, 12 ldc (HER2K); the lowest-numbered illegal argument wins.
int check_her(int order, int uplo, int trans, int N, int K, int lda, int ldb, int ldc, bool two) {
    const bool rows_n = (trans == NoTrans) != (order == CblasRowMajor);
    const int nrowa = rows_n ? N : K;
    auto mx1 = [](int v) { return v > 1 ? v : 1; };
    if (!to_uplo(uplo)) return 1;
    if (trans != NoTrans && trans != ConjT) return 2;
    if (N < 0) return 3;
    if (K < 0) return 4;
    if (lda < mx1(nrowa)) return 7;
    if (two && ldb < mx1(nrowa)) return 9;
    if (ldc < mx1(N)) return two ? 12 : 10;
    return 0;
}

// op(X) op(Y)^H as a column-major GEMM with a triangular, Hermitian output.
// A row-major call is the column-major one on the transposes: with C^T =
// conj(C), the triangle flips and NoTrans / ConjTrans swap.
Gemm herm_gemm(DType dt, int order, int uplo, int trans, int N, int K, cplx alpha, const void *X, int ldx,
               const void *Y, int ldy, cplx beta, void *C, int ldc) {
    int u = to_uplo(uplo);
    bool ct = trans == ConjT;
    if (order == CblasRowMajor) {
        u = 3 - u;
        ct = !ct;
    }
    Gemm g;
    g.dt = dt;
    g.M = N; g.N = N; g.K = K;
    g.ta = ct ? ConjT : NoTrans;  // op(X): N x K
    g.tb = ct ? NoTrans : ConjT;  // op(Y)^H: K x N
    g.A = X; g.lda = ldx;
    g.B = Y; g.ldb = ldy;
    g.alpha = alpha; g.beta = beta;
    g.C = C; g.ldc = ldc;
    g.uplo = u;
    g.diag = 0;
    g.herm_out = true;
    return g;
}

void herk_entry(const char *name, DType dt, int order, int uplo, int trans, int N, int K, double alpha,
                const void *A, int lda, double beta, void *C, int ldc) {
    clear_error();
    int info = check_her(order, uplo, trans, N, K, lda, 0, ldc, false);
    if (info) {
        set_error(BLASX_ERR_ARG, "%s parameter %d illegal", name, info);
        xerbla_(const_cast<char *>(name), &info);
        return;
    }
    if (N == 0) return;
    host_gemm(herm_gemm(dt, order, uplo, trans, N, K, cplx{alpha, 0.0}, A, lda, A, lda, cplx{beta, 0.0}, C, ldc));
}

// C = alpha op(A) op(B)^H + conj(alpha) op(B) op(A)^H + beta C: two Hermitian
// triangular GEMMs, the second accumulating onto the first.
void her2k_entry(const char *name, DType dt, int order, int uplo, int trans, int N, int K, cplx alpha,
                 const void *A, int lda, const void *B, int ldb, double beta, void *C, int ldc) {
    clear_error();
    int info = check_her(order, uplo, trans, N, K, lda, ldb, ldc, true);
    if (info) {
        set_error(BLASX_ERR_ARG, "%s parameter %d illegal", name, info);
        xerbla_(const_cast<char *>(name), &info);
        return;
    }
    if (N == 0) return;
    // row-major: C^T = conj(alpha) op'(A) op'(B)^H + alpha op'(B) op'(A)^H + beta C^T
    // on the column-major views (herm_gemm flips uplo and trans)
    if (order == CblasRowMajor) alpha.im = -alpha.im;
    host_gemm(herm_gemm(dt, order, uplo, trans, N, K, alpha, A, lda, B, ldb, cplx{beta, 0.0}, C, ldc));
    if (last_status() != BLASX_OK) return;
    if (alpha.re == 0 && alpha.im == 0) return;  // the first call already scaled C by beta
    host_gemm(herm_gemm(dt, order, uplo, trans, N, K, cplx{alpha.re, -alpha.im}, B, ldb, A, lda, cplx{1.0, 0.0}, C,
                        ldc));
}

bool f77_uplo(const char *c, int *u) {
    switch (*c) {
        case 'U': case 'u': *u = CblasUpper; return true;
        case 'L': case 'l': *u = CblasLower; return true;
        default: return false;
    }
}
bool f77_trans1(const char *c, int *t) {
    switch (*c) {
        case 'N': case 'n': *t = NoTrans; return true;
        case 'T': case 't': *t = TransT; return true;
        case 'C': case 'c': *t = ConjT; return true;
        default: return false;
    }
}

}  // namespace

int syrk_device(DType dt, int uplo, int trans, int N, int K, cplx alpha, const void *A, int lda,
                cplx beta, void *C, int ldc, cudaStream_t s) {
    clear_error();
    const int info = check_syr(dt, CblasColMajor, uplo, trans, N, K, lda, 0, ldc, false);
    if (info) return set_error(BLASX_ERR_ARG, "device syrk parameter %d illegal", info);
    if (N == 0) return BLASX_OK;
    Context *c = context();
    if (!c) return last_status();
    const Gemm g = tri_gemm(dt, CblasColMajor, uplo, trans, N, K, alpha, A, lda, A, lda, beta, C, ldc);
    if (g.alpha_zero() || g.K == 0) return launch_scale(g, s);
    return device_gemm(g, s);
}

}  // namespace bx

using bx::cplx;
using bx::DType;

extern "C" {

void cblas_ssyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const float alpha,
                 const float *A, const int lda, const float beta, float *C, const int ldc) {
    bx::syrk_entry("SSYRK ", DType::F32, Order, Uplo, Trans, N, K, cplx{alpha, 0}, A, lda,
                   cplx{beta, 0}, C, ldc);
}

void cblas_dsyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                 const double *A, const int lda, const double beta, double *C, const int ldc) {
    bx::syrk_entry("DSYRK ", DType::F64, Order, Uplo, Trans, N, K, cplx{alpha, 0}, A, lda,
                   cplx{beta, 0}, C, ldc);
}

void cblas_zsyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                 const void *A, const int lda, const void *beta, void *C, const int ldc) {
    const double *al = static_cast<const double *>(alpha);
    const double *be = static_cast<const double *>(beta);
    bx::syrk_entry("ZSYRK ", DType::C128, Order, Uplo, Trans, N, K, cplx{al[0], al[1]}, A, lda,
                   cplx{be[0], be[1]}, C, ldc);
}

void cblas_ssyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const float alpha,
                  const float *A, const int lda, const float *B, const int ldb, const float beta,
                  float *C, const int ldc) {
    bx::syr2k_entry("SSYR2K", DType::F32, Order, Uplo, Trans, N, K, cplx{alpha, 0}, A, lda, B, ldb,
                    cplx{beta, 0}, C, ldc);
}

void cblas_dsyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                  const double *A, const int lda, const double *B, const int ldb, const double beta,
                  double *C, const int ldc) {
    bx::syr2k_entry("DSYR2K", DType::F64, Order, Uplo, Trans, N, K, cplx{alpha, 0}, A, lda, B, ldb,
                    cplx{beta, 0}, C, ldc);
}

void cblas_zsyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const void *beta,
                  void *C, const int ldc) {
    const double *al = static_cast<const double *>(alpha);
    const double *be = static_cast<const double *>(beta);
    bx::syr2k_entry("ZSYR2K", DType::C128, Order, Uplo, Trans, N, K, cplx{al[0], al[1]}, A, lda, B,
                    ldb, cplx{be[0], be[1]}, C, ldc);
}

void cblas_csyrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                 const void *A, const int lda, const void *beta, void *C, const int ldc) {
    const float *al = static_cast<const float *>(alpha);
    const float *be = static_cast<const float *>(beta);
    bx::syrk_entry("CSYRK ", DType::C64, Order, Uplo, Trans, N, K, cplx{al[0], al[1]}, A, lda,
                   cplx{be[0], be[1]}, C, ldc);
}

void cblas_csyr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const void *beta,
                  void *C, const int ldc) {
    const float *al = static_cast<const float *>(alpha);
    const float *be = static_cast<const float *>(beta);
    bx::syr2k_entry("CSYR2K", DType::C64, Order, Uplo, Trans, N, K, cplx{al[0], al[1]}, A, lda, B,
                    ldb, cplx{be[0], be[1]}, C, ldc);
}

// CHERK / ZHERK report as "CHERK" / "ZHERK", CHER2K as "CHER2K" and ZHER2K as
// "ZHERK", the names the reference passes to xerbla_ (blas/cherk.c:13,
// blas/zherk.c:13, blas/cher2k.c:13, blas/zher2k.c:13).
void cblas_cherk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const float alpha,
                 const void *A, const int lda, const float beta, void *C, const int ldc) {
    bx::herk_entry("CHERK", DType::C64, Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc);
}

void cblas_zherk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                 const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const double alpha,
                 const void *A, const int lda, const double beta, void *C, const int ldc) {
    bx::herk_entry("ZHERK", DType::C128, Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc);
}

void cblas_cher2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const float beta,
                  void *C, const int ldc) {
    const float *al = static_cast<const float *>(alpha);
    bx::her2k_entry("CHER2K", DType::C64, Order, Uplo, Trans, N, K, cplx{al[0], al[1]}, A, lda, B, ldb, beta, C,
                    ldc);
}

void cblas_zher2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,
                  const enum CBLAS_TRANSPOSE Trans, const int N, const int K, const void *alpha,
                  const void *A, const int lda, const void *B, const int ldb, const double beta,
                  void *C, const int ldc) {
    const double *al = static_cast<const double *>(alpha);
    bx::her2k_entry("ZHERK", DType::C128, Order, Uplo, Trans, N, K, cplx{al[0], al[1]}, A, lda, B, ldb, beta, C,
                    ldc);
}

// F77 wrappers: a bad Trans overrides a bad Uplo (blas/dsyrk.c:86-91).
#define BX_F77_SYR_PROLOGUE(NAME)                                        \
    int up = 0, tr = 0, info = -1;                                       \
    if (!bx::f77_uplo(uplo, &up)) info = 1;                              \
    if (!bx::f77_trans1(trans, &tr)) info = 2;                           \
    if (info >= 0) {                                                     \
        bx::set_error(BLASX_ERR_ARG, "%s parameter %d illegal", NAME, info); \
        xerbla_(const_cast<char *>(NAME), &info);                        \
        return;                                                          \
    }

void ssyrk_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda,
            float *beta, float *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("SSYRK ")
    cblas_ssyrk(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, *alpha, A, *lda, *beta,
                C, *ldc);
}

void dsyrk_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
            double *beta, double *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("DSYRK ")
    cblas_dsyrk(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, *alpha, A, *lda, *beta,
                C, *ldc);
}

void zsyrk_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
            double *beta, double *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("ZSYRK ")
    cblas_zsyrk(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, alpha, A, *lda, beta, C,
                *ldc);
}

void ssyr2k_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *B,
             int *ldb, float *beta, float *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("SSYR2K")
    cblas_ssyr2k(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, *alpha, A, *lda, B,
                 *ldb, *beta, C, *ldc);
}

void dsyr2k_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
             double *B, int *ldb, double *beta, double *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("DSYR2K")
    cblas_dsyr2k(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, *alpha, A, *lda, B,
                 *ldb, *beta, C, *ldc);
}

void zsyr2k_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda,
             double *B, int *ldb, double *beta, double *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("ZSYR2K")
    cblas_zsyr2k(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, alpha, A, *lda, B,
                 *ldb, beta, C, *ldc);
}

void csyrk_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *beta,
            float *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("CSYRK ")
    cblas_csyrk(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, alpha, A, *lda, beta, C, *ldc);
}

void csyr2k_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *B,
             int *ldb, float *beta, float *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("CSYR2K")
    cblas_csyr2k(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, alpha, A, *lda, B, *ldb,
                 beta, C, *ldc);
}

// F77 HERK / HER2K: real alpha (HERK) and beta by pointer, complex alpha of
// HER2K as an (re, im) pair (blas/zherk.c:81-104, blas/zher2k.c:89-118).
void cherk_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *beta,
            float *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("CHERK")
    cblas_cherk(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, *alpha, A, *lda, *beta, C, *ldc);
}

void zherk_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda, double *beta,
            double *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("ZHERK")
    cblas_zherk(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, *alpha, A, *lda, *beta, C, *ldc);
}

void cher2k_(char *uplo, char *trans, int *n, int *k, float *alpha, float *A, int *lda, float *B, int *ldb,
             float *beta, float *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("CHER2K")
    cblas_cher2k(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, alpha, A, *lda, B, *ldb, *beta, C,
                 *ldc);
}

void zher2k_(char *uplo, char *trans, int *n, int *k, double *alpha, double *A, int *lda, double *B,
             int *ldb, double *beta, double *C, int *ldc) {
    BX_F77_SYR_PROLOGUE("ZHERK")
    cblas_zher2k(CblasColMajor, CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), *n, *k, alpha, A, *lda, B, *ldb, *beta, C,
                 *ldc);
}

int blasx_dsyrk_device(int uplo, int trans, int N, int K, double alpha, const double *A, int lda,
                       double beta, double *C, int ldc, void *stream) {
    return bx::syrk_device(DType::F64, uplo, trans, N, K, cplx{alpha, 0}, A, lda, cplx{beta, 0}, C,
                           ldc, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
