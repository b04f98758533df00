// symm_trmm_api.cu -- cblas_?symm, cblas_?hemm, cblas_?trmm, cblas_?trsm and
// their F77 wrappers on the GPU.
//
// The reference declares these but always runs them on its host BLAS (for
// instance blas/dsymm.c:44-57 and blas/dtrmm.c:49-60 select the CPU in every
// branch of their dispatchers). Here:
//   SYMM / HEMM  C = alpha A B + beta C (side Left, A is M x M) or
//                C = alpha B A + beta C (side Right, A is N x N): a GEMM
//                whose square operand is stored as one triangle; the host
//                path completes it on the device (mirror, or conjugate
//                mirror) and runs the product on the native or emulated path
//                like any GEMM, in or out of core.
//   TRMM         B = alpha op(A) B (Left) or alpha B op(A) (Right), in place
//                (trsm.cu: recursive halving into GEMM updates and leaves
//                that multiply by their completed diagonal block).
//   TRSM         solves op(A) X = alpha B (Left) or X op(A) = alpha B (Right)
//                for X, which overwrites B (trsm.cu: recursive halving into
//                GEMM updates and a substitution kernel).
// Row-major calls are the column-major problem with side and uplo flipped and
// M, N swapped (the reference ignores Order).
//
// Argument checks follow the reference's order (blas/dsymm.c:29-36,
// blas/dtrmm.c:32-40): the first illegal argument is reported through xerbla_
// -- SYMM / HEMM: 1 Side, 2 Uplo, 3 M, 4 N, 7 lda, 9 ldb, 12 ldc; TRMM: 1 Side,
// 2 Uplo, 3 TransA, 4 Diag, 5 M, 6 N, 9 lda, 11 ldb; TRSM the same codes
// (blas/dtrsm.c:31-38). The F77 wrappers report
// the first bad character argument likewise (blas/dsymm.c:83-84,
// blas/dtrmm.c:76-80). CHEMM / ZHEMM report under the reference's names
// "CHEMM" / "ZHEMM", without the trailing blank (blas/zhemm.c:14).
#include <algorithm>

#include "host_pipeline.h"
#include "kernels.h"
#include "runtime.h"

namespace bx {
namespace {

bool side_ok(int s) { return s == CblasLeft || s == CblasRight; }
bool uplo_ok(int u) { return u == CblasUpper || u == CblasLower; }
bool diag_ok(int d) { return d == CblasNonUnit || d == CblasUnit; }
bool trans_ok(int t) { return t == NoTrans || t == TransT || t == ConjT; }
int flip_side(int s) { return s == CblasLeft ? CblasRight : CblasLeft; }
int flip_uplo(int u) { return u == CblasUpper ? CblasLower : CblasUpper; }

void report(const char *name, int info) {
    set_error(BLASX_ERR_ARG, "%s parameter %d illegal", name, info);
    xerbla_(const_cast<char *>(name), &info);
}

// Column-major symm / hemm (side, uplo, M, N already column-major; M, N >= 0).
void symm_col(const char *name, DType dt, bool herm, int side, int uplo, int M, int N, cplx alpha,
              const void *A, int lda, const void *B, int ldb, cplx beta, void *C, int ldc) {
    int info = 0;
    const int nrowa = side == CblasLeft ? M : N;
    auto mx1 = [](int v) { return v > 1 ? v : 1; };
    if (lda < mx1(nrowa)) info = 7;
    else if (ldb < mx1(M)) info = 9;
    else if (ldc < mx1(M)) info = 12;
    if (info) return report(name, info);
    if (M == 0 || N == 0) return;
    const int form = herm ? (uplo == CblasUpper ? kHermUpper : kHermLower)
                          : (uplo == CblasUpper ? kSymUpper : kSymLower);
    Gemm g;
    g.dt = dt;
    g.ta = NoTrans; g.tb = NoTrans;
    g.M = M; g.N = N;
    if (side == CblasLeft) {
        g.K = M;
        g.A = A; g.lda = lda; g.B = B; g.ldb = ldb;
        g.a_form = form;
    } else {
        g.K = N;
        g.A = B; g.lda = ldb; g.B = A; g.ldb = lda;
        g.b_form = form;
    }
    g.alpha = alpha; g.beta = beta;
    g.C = C; g.ldc = ldc;
    host_gemm(g);
}

void symm_entry(const char *name, DType dt, bool herm, int order, int side, int uplo, int M, int N,
                cplx alpha, const void *A, int lda, const void *B, int ldb, cplx beta, void *C,
                int ldc) {
    clear_error();
    if (!side_ok(side)) return report(name, 1);
    if (!uplo_ok(uplo)) return report(name, 2);
    if (M < 0) return report(name, 3);
    if (N < 0) return report(name, 4);
    if (order == CblasRowMajor)
        return symm_col(name, dt, herm, flip_side(side), flip_uplo(uplo), N, M, alpha, A, lda, B, ldb,
                        beta, C, ldc);
    symm_col(name, dt, herm, side, uplo, M, N, alpha, A, lda, B, ldb, beta, C, ldc);
}

void trmm_col(const char *name, DType dt, int side, int uplo, int trans, int diag, int M, int N,
              cplx alpha, const void *A, int lda, void *B, int ldb) {
    int info = 0;
    const int nrowa = side == CblasLeft ? M : N;
    auto mx1 = [](int v) { return v > 1 ? v : 1; };
    if (lda < mx1(nrowa)) info = 9;
    else if (ldb < mx1(M)) info = 11;
    if (info) return report(name, info);
    if (M == 0 || N == 0) return;
    Trsm t;
    t.dt = dt;
    t.left = side == CblasLeft;
    t.lower = uplo == CblasLower;
    t.unit = diag == CblasUnit;
    t.trans = (!is_complex(dt) && trans == ConjT) ? TransT : trans;
    t.M = M; t.N = N;
    t.alpha = alpha;
    t.A = A; t.lda = lda;
    t.B = B; t.ldb = ldb;
    host_trmm(t);
}

void trmm_entry(const char *name, DType dt, int order, int side, int uplo, int trans, int diag, int M,
                int N, cplx alpha, const void *A, int lda, void *B, int ldb) {
    clear_error();
    if (!side_ok(side)) return report(name, 1);
    if (!uplo_ok(uplo)) return report(name, 2);
    if (!trans_ok(trans)) return report(name, 3);
    if (!diag_ok(diag)) return report(name, 4);
    if (M < 0) return report(name, 5);
    if (N < 0) return report(name, 6);
    if (order == CblasRowMajor)
        return trmm_col(name, dt, flip_side(side), flip_uplo(uplo), trans, diag, N, M, alpha, A, lda, B, ldb);
    trmm_col(name, dt, side, uplo, trans, diag, M, N, alpha, A, lda, B, ldb);
}

void trsm_col(const char *name, DType dt, int side, int uplo, int trans, int diag, int M, int N,
              cplx alpha, const void *A, int lda, void *B, int ldb) {
    int info = 0;
    const int nrowa = side == CblasLeft ? M : N;
    auto mx1 = [](int v) { return v > 1 ? v : 1; };
    if (lda < mx1(nrowa)) info = 9;
    else if (ldb < mx1(M)) info = 11;
    if (info) return report(name, info);
    if (M == 0 || N == 0) return;
    Trsm t;
    t.dt = dt;
    t.left = side == CblasLeft;
    t.lower = uplo == CblasLower;
    t.unit = diag == CblasUnit;
    t.trans = (!is_complex(dt) && trans == ConjT) ? TransT : trans;
    t.M = M; t.N = N;
    t.alpha = alpha;
    t.A = A; t.lda = lda;
    t.B = B; t.ldb = ldb;
    host_trsm(t);
}

void trsm_entry(const char *name, DType dt, int order, int side, int uplo, int trans, int diag, int M,
                int N, cplx alpha, const void *A, int lda, void *B, int ldb) {
    clear_error();
    if (!side_ok(side)) return report(name, 1);
    if (!uplo_ok(uplo)) return report(name, 2);
    if (!trans_ok(trans)) return report(name, 3);
    if (!diag_ok(diag)) return report(name, 4);
    if (M < 0) return report(name, 5);
    if (N < 0) return report(name, 6);
    if (order == CblasRowMajor)
        return trsm_col(name, dt, flip_side(side), flip_uplo(uplo), trans, diag, N, M, alpha, A, lda, B, ldb);
    trsm_col(name, dt, side, uplo, trans, diag, M, N, alpha, A, lda, B, ldb);
}

bool f77_side(const char *c, int *s) {
    switch (*c) {
        case 'L': case 'l': *s = CblasLeft; return true;
        case 'R': case 'r': *s = CblasRight; return true;
        default: return false;
    }
}
bool f77_uplo2(const char *c, int *u) {
    switch (*c) {
        case 'U': case 'u': *u = CblasUpper; return true;
        case 'L': case 'l': *u = CblasLower; return true;
        default: return false;
    }
}
bool f77_trans2(const char *c, int *t) {
    switch (*c) {
        case 'N': case 'n': *t = NoTrans; return true;
        case 'T': case 't': *t = TransT; return true;
        case 'C': case 'c': *t = ConjT; return true;
        default: return false;
    }
}
bool f77_diag(const char *c, int *d) {
    switch (*c) {
        case 'N': case 'n': *d = CblasNonUnit; return true;
        case 'U': case 'u': *d = CblasUnit; return true;
        default: return false;
    }
}

cplx real_scalar(double v) { return cplx{v, 0.0}; }
cplx z_scalar(const void *p) {
    const double *d = static_cast<const double *>(p);
    return cplx{d[0], d[1]};
}
cplx c_scalar(const void *p) {
    const float *f = static_cast<const float *>(p);
    return cplx{f[0], f[1]};
}

}  // namespace

// Device-resident TRSM (mult false) or TRMM (mult true) on the caller's
// stream. TRMM's leaf scratch (one diagonal block, one leaf's vectors) is a
// stream-ordered allocation on that stream, released after the last leaf.
int tri_device_entry(bool mult, DType dt, int side, int uplo, int trans, int diag, int M, int N, cplx alpha,
                     const void *A, int lda, void *B, int ldb, cudaStream_t s) {
    clear_error();
    int info = 0;
    const int nrowa = side == CblasLeft ? M : N;
    if (!side_ok(side)) info = 1;
    else if (!uplo_ok(uplo)) info = 2;
    else if (!trans_ok(trans)) info = 3;
    else if (!diag_ok(diag)) info = 4;
    else if (M < 0) info = 5;
    else if (N < 0) info = 6;
    else if (lda < std::max(1, nrowa)) info = 9;
    else if (ldb < std::max(1, M)) info = 11;
    if (info) return set_error(BLASX_ERR_ARG, "device %s parameter %d illegal", mult ? "trmm" : "trsm", info);
    if (M == 0 || N == 0) return BLASX_OK;
    if (!context()) return last_status();
    Trsm t;
    t.dt = dt;
    t.left = side == CblasLeft;
    t.lower = uplo == CblasLower;
    t.unit = diag == CblasUnit;
    t.trans = (!is_complex(dt) && trans == ConjT) ? TransT : trans;
    t.M = M; t.N = N;
    t.alpha = alpha;
    t.A = A; t.lda = lda;
    t.B = B; t.ldb = ldb;
    bool emulated = false;
    if (!mult) return trsm_device(t, s, &emulated);
    TrmmScratch w = trmm_scratch_sizes(t);
    BX_CUDA(dev_malloc_async(&w.diag, w.diag_bytes, s));
    if (dev_malloc_async(&w.temp, w.temp_bytes, s) != cudaSuccess) {
        cudaFreeAsync(w.diag, s);
        return set_error(BLASX_ERR_NOMEM, "device trmm: no memory for %zu bytes of scratch", w.temp_bytes);
    }
    const int rc = trmm_device(t, w, s, &emulated);
    cudaFreeAsync(w.temp, s);
    cudaFreeAsync(w.diag, s);
    return rc;
}

}  // namespace bx

using bx::cplx;
using bx::DType;

extern "C" {

#define BX_SYMM(NAME, CNAME, DT, HERM, STYPE, ET, TOSC)                                                 \
    void CNAME(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side, const enum CBLAS_UPLO Uplo,     \
               const int M, const int N, STYPE alpha, const ET *A, const int lda, const ET *B,           \
               const int ldb, STYPE beta, ET *C, const int ldc) {                                       \
        bx::symm_entry(NAME, DT, HERM, Order, Side, Uplo, M, N, TOSC(alpha), A, lda, B, ldb, TOSC(beta), \
                       C, ldc);                                                                         \
    }

BX_SYMM("SSYMM ", cblas_ssymm, DType::F32, false, const float, float, bx::real_scalar)
BX_SYMM("DSYMM ", cblas_dsymm, DType::F64, false, const double, double, bx::real_scalar)
BX_SYMM("CSYMM ", cblas_csymm, DType::C64, false, const void *, void, bx::c_scalar)
BX_SYMM("ZSYMM ", cblas_zsymm, DType::C128, false, const void *, void, bx::z_scalar)
BX_SYMM("CHEMM", cblas_chemm, DType::C64, true, const void *, void, bx::c_scalar)
BX_SYMM("ZHEMM", cblas_zhemm, DType::C128, true, const void *, void, bx::z_scalar)
#undef BX_SYMM

#define BX_TRMM(NAME, CNAME, DT, STYPE, ET, TOSC)                                                       \
    void CNAME(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side, const enum CBLAS_UPLO Uplo,     \
               const enum CBLAS_TRANSPOSE TransA, const enum CBLAS_DIAG Diag, const int M, const int N,  \
               STYPE alpha, const ET *A, const int lda, ET *B, const int ldb) {                         \
        bx::trmm_entry(NAME, DT, Order, Side, Uplo, TransA, Diag, M, N, TOSC(alpha), A, lda, B, ldb);   \
    }

BX_TRMM("STRMM ", cblas_strmm, DType::F32, const float, float, bx::real_scalar)
BX_TRMM("DTRMM ", cblas_dtrmm, DType::F64, const double, double, bx::real_scalar)
BX_TRMM("CTRMM ", cblas_ctrmm, DType::C64, const void *, void, bx::c_scalar)
BX_TRMM("ZTRMM ", cblas_ztrmm, DType::C128, const void *, void, bx::z_scalar)
#undef BX_TRMM

#define BX_TRSM(NAME, CNAME, DT, STYPE, ET, TOSC)                                                       \
    void CNAME(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side, const enum CBLAS_UPLO Uplo,     \
               const enum CBLAS_TRANSPOSE TransA, const enum CBLAS_DIAG Diag, const int M, const int N,  \
               STYPE alpha, const ET *A, const int lda, ET *B, const int ldb) {                         \
        bx::trsm_entry(NAME, DT, Order, Side, Uplo, TransA, Diag, M, N, TOSC(alpha), A, lda, B, ldb);   \
    }

BX_TRSM("STRSM ", cblas_strsm, DType::F32, const float, float, bx::real_scalar)
BX_TRSM("DTRSM ", cblas_dtrsm, DType::F64, const double, double, bx::real_scalar)
BX_TRSM("CTRSM ", cblas_ctrsm, DType::C64, const void *, void, bx::c_scalar)
BX_TRSM("ZTRSM ", cblas_ztrsm, DType::C128, const void *, void, bx::z_scalar)
#undef BX_TRSM

// F77 wrappers. Scalars by pointer: one real for S/D, an (re, im) pair for C/Z.
#define BX_F77_SYMM(NAME, FNAME, CNAME, RT, SCAL)                                                      \
    void FNAME(char *side, char *uplo, int *m, int *n, RT *alpha, RT *A, int *lda, RT *B, int *ldb,     \
               RT *beta, RT *C, int *ldc) {                                                             \
        int sd = 0, up = 0, info = 0;                                                                  \
        if (!bx::f77_uplo2(uplo, &up)) info = 2;                                                       \
        if (!bx::f77_side(side, &sd)) info = 1;                                                        \
        if (info) return bx::report(NAME, info);                                                       \
        CNAME(CblasColMajor, CBLAS_SIDE(sd), CBLAS_UPLO(up), *m, *n, SCAL(alpha), A, *lda, B, *ldb,     \
              SCAL(beta), C, *ldc);                                                                     \
    }
#define BX_REAL(p) (*(p))
#define BX_PTR(p) (p)
BX_F77_SYMM("SSYMM ", ssymm_, cblas_ssymm, float, BX_REAL)
BX_F77_SYMM("DSYMM ", dsymm_, cblas_dsymm, double, BX_REAL)
BX_F77_SYMM("CSYMM ", csymm_, cblas_csymm, float, BX_PTR)
BX_F77_SYMM("ZSYMM ", zsymm_, cblas_zsymm, double, BX_PTR)
BX_F77_SYMM("CHEMM", chemm_, cblas_chemm, float, BX_PTR)
BX_F77_SYMM("ZHEMM", zhemm_, cblas_zhemm, double, BX_PTR)
#undef BX_F77_SYMM

#define BX_F77_TRI(NAME, FNAME, CNAME, RT, SCAL)                                                      \
    void FNAME(char *side, char *uplo, char *transa, char *diag, int *m, int *n, RT *alpha, RT *A,      \
               int *lda, RT *B, int *ldb) {                                                             \
        int sd = 0, up = 0, tr = 0, dg = 0, info = 0;                                                  \
        if (!bx::f77_diag(diag, &dg)) info = 4;                                                        \
        if (!bx::f77_trans2(transa, &tr)) info = 3;                                                    \
        if (!bx::f77_uplo2(uplo, &up)) info = 2;                                                       \
        if (!bx::f77_side(side, &sd)) info = 1;                                                        \
        if (info) return bx::report(NAME, info);                                                       \
        CNAME(CblasColMajor, CBLAS_SIDE(sd), CBLAS_UPLO(up), CBLAS_TRANSPOSE(tr), CBLAS_DIAG(dg), *m, *n, \
              SCAL(alpha), A, *lda, B, *ldb);                                                           \
    }
BX_F77_TRI("STRMM ", strmm_, cblas_strmm, float, BX_REAL)
BX_F77_TRI("DTRMM ", dtrmm_, cblas_dtrmm, double, BX_REAL)
BX_F77_TRI("CTRMM ", ctrmm_, cblas_ctrmm, float, BX_PTR)
BX_F77_TRI("ZTRMM ", ztrmm_, cblas_ztrmm, double, BX_PTR)
BX_F77_TRI("STRSM ", strsm_, cblas_strsm, float, BX_REAL)
BX_F77_TRI("DTRSM ", dtrsm_, cblas_dtrsm, double, BX_REAL)
BX_F77_TRI("CTRSM ", ctrsm_, cblas_ctrsm, float, BX_PTR)
BX_F77_TRI("ZTRSM ", ztrsm_, cblas_ztrsm, double, BX_PTR)
#undef BX_F77_TRI

int blasx_dtrsm_device(int side, int uplo, int trans, int diag, int M, int N, double alpha, const double *A,
                       int lda, double *B, int ldb, void *stream) {
    return bx::tri_device_entry(false, DType::F64, side, uplo, trans, diag, M, N, cplx{alpha, 0.0}, A, lda, B, ldb,
                                static_cast<cudaStream_t>(stream));
}

int blasx_dtrmm_device(int side, int uplo, int trans, int diag, int M, int N, double alpha, const double *A,
                       int lda, double *B, int ldb, void *stream) {
    return bx::tri_device_entry(true, DType::F64, side, uplo, trans, diag, M, N, cplx{alpha, 0.0}, A, lda, B, ldb,
                                static_cast<cudaStream_t>(stream));
}
#undef BX_REAL
#undef BX_PTR

}  // extern "C"
