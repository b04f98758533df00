/* Links a C program against libblasx_b200.so the way a BLASX user links
 * -lblasx: a cblas.h-style header first (guarded by CBLAS_H, as the
 * reference's), then blasx_b200.h. Exercises calls that need no GPU. */
#include <stdio.h>

#ifndef CBLAS_H
#define CBLAS_H
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
#endif
#include "blasx_b200.h"

int main(void) {
    double A[16] = {0}, B[16] = {0}, C[16];
    for (int i = 0; i < 16; ++i) C[i] = 1.0;
    /* lda = 2 < M = 4: parameter 8 */
    cblas_dgemm(CblasColMajor, CblasNoTrans, CblasNoTrans, 4, 4, 4, 1.0, A, 2, B, 4, 0.0, C, 4);
    fflush(stdout);
    printf("status=%d\n", blasx_last_status());
    /* F77: bad transa */
    char ta = 'X', tb = 'N';
    int m = 4, n = 4, k = 4, ld = 4;
    double al = 1.0, be = 0.0;
    dgemm_(&ta, &tb, &m, &n, &k, &al, A, &ld, B, &ld, &be, C, &ld);
    fflush(stdout);
    /* DSYRK: ldc = 2 < N = 4: parameter 10 */
    cblas_dsyrk(CblasColMajor, CblasUpper, CblasNoTrans, 4, 4, 1.0, A, 4, 0.0, C, 2);
    fflush(stdout);
    /* DSYMM: ldb = 2 < M = 4: parameter 9; ZHEMM: bad side; DTRMM: bad diag */
    cblas_dsymm(CblasColMajor, CblasLeft, CblasUpper, 4, 4, 1.0, A, 4, B, 2, 0.0, C, 4);
    fflush(stdout);
    double one[2] = {1.0, 0.0};
    cblas_zhemm(CblasColMajor, (enum CBLAS_SIDE)0, CblasUpper, 2, 2, one, A, 2, B, 2, one, C, 2);
    fflush(stdout);
    cblas_dtrmm(CblasColMajor, CblasRight, CblasLower, CblasTrans, (enum CBLAS_DIAG)7, 4, 4, 1.0, A, 4, C, 4);
    fflush(stdout);
    /* DTRSM: ldb = 2 < M = 4: parameter 11; F77 dtrsm_: bad side */
    cblas_dtrsm(CblasColMajor, CblasLeft, CblasUpper, CblasNoTrans, CblasNonUnit, 4, 4, 1.0, A, 4, C, 2);
    fflush(stdout);
    char sd = 'X', up = 'U', tn = 'N', dg = 'N';
    dtrsm_(&sd, &up, &tn, &dg, &m, &n, &al, A, &ld, C, &ld);
    fflush(stdout);
    /* M = 0: quick return, no device needed */
    cblas_dgemm(CblasColMajor, CblasNoTrans, CblasNoTrans, 0, 4, 4, 1.0, A, 4, B, 4, 0.0, C, 4);
    printf("status=%d C0=%g\n", blasx_last_status(), C[0]);
    blasx_tile_plan_stats st;
    int rc = blasx_tile_plan(40960, 40960, 40960, 4096, 24LL << 30, 8, 0, &st);
    printf("plan rc=%d loads=%lld min_ratio=%.3f\n", rc, st.tile_loads,
           st.operand_h2d_bytes / st.min_operand_h2d_bytes);
    return 0;
}
