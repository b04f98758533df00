// host_pipeline.h -- GEMM on host-resident operands: staging into HBM,
// device compute and write-back of C.
#pragma once

#include "runtime.h"

namespace bx {

// Runs a column-major GEMM whose A, B, C are host pointers. Synchronous: C is
// complete on return. Records status and call statistics for the thread.
int host_gemm(const Gemm &g);

// Triangular solve (TRSM) whose A and B are host pointers; synchronous, B
// holds the solution on return. In core only (BLASX_ERR_UNSUPPORTED beyond
// the HBM budget, B unchanged).
int host_trsm(const Trsm &t);
// Triangular multiply (TRMM: B = alpha op(A) B or alpha B op(A), described by
// a Trsm), host pointers, synchronous, in core only like host_trsm.
int host_trmm(const Trsm &t);

}  // namespace bx
