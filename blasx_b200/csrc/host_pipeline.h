// host_pipeline.h -- GEMM on host-resident operands: staging into HBM,
// device compute and write-back of C.
#pragma once

#include "runtime.h"

namespace bx {

// Runs a column-major GEMM whose A, B, C are host pointers. Synchronous: C is
// complete on return. Records status and call statistics for the thread.
int host_gemm(const Gemm &g);

}  // namespace bx
