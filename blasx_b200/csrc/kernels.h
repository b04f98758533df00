// kernels.h -- device-side entry points of the GEMM kernels. All pointers are
// device addresses, column-major, leading dimensions in elements.
#pragma once

#include "runtime.h"

namespace bx {

// C = beta * C (alpha == 0 or K == 0); C is not read when beta == 0.
int launch_scale(const Gemm &g, cudaStream_t s);

// Portable SIMT tiled kernel (all dtypes, transposes, ragged edges). Used for
// small problems and as the first correct path.
int launch_gemm_simt(const Gemm &g, cudaStream_t s);

// Native FP64 / complex128 kernel on the FP64 tensor pipe (DMMA).
int launch_gemm_dmma(const Gemm &g, cudaStream_t s);
bool dmma_supported(const Gemm &g);

// Device-resident GEMM of any dtype through the best available path.
// Uses library-owned scratch memory for the Ozaki path.
int device_gemm(const Gemm &g, cudaStream_t s);

}  // namespace bx
