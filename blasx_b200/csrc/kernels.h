// kernels.h -- device-side entry points of the GEMM kernels. All pointers are
// device addresses, column-major, leading dimensions in elements.
#pragma once

#include "runtime.h"

namespace bx {

// C = beta * C (alpha == 0 or K == 0); C is not read when beta == 0.
int launch_scale(const Gemm &g, cudaStream_t s);
// Completes the n x n operand X (ld ldx, device, in place) from its stored
// triangle according to `form` (an OperandForm): mirror, conjugate-mirror, or
// zero the other triangle (and set a unit diagonal). Entries of the stored
// triangle are only read, except Hermitian diagonals (imaginary part set to
// zero) and unit diagonals (set to one).
int launch_complete_operand(DType dt, int form, void *X, int64_t ldx, int64_t n, cudaStream_t s);
// Zeroes the imaginary parts of the entries (r, c) of the m x n device block
// C (ld ldc) with r - c == off; nothing for real types.
int launch_real_diagonal(DType dt, void *C, int64_t ldc, int64_t m, int64_t n, int64_t off, cudaStream_t s);
// g.C (g.M x g.N, ld g.ldc) += g.beta * X (ld ldx); nothing when beta == 0.
int launch_add_scaled(const Gemm &g, const void *X, int64_t ldx, cudaStream_t s);

// Portable SIMT tiled kernel (all dtypes, transposes, ragged edges). Used for
// small problems and as the first correct path.
int launch_gemm_simt(const Gemm &g, cudaStream_t s);

// Native FP64 / complex128 kernel on the FP64 tensor pipe (DMMA).
int launch_gemm_dmma(const Gemm &g, cudaStream_t s);
bool dmma_supported(const Gemm &g);


// Device-resident GEMM of any dtype through the best available path.
// Uses library-owned scratch memory for the Ozaki path.
int device_gemm(const Gemm &g, cudaStream_t s);
// FP32 on the CUDA cores with a 128 x 128 tile per CTA, for problems of at
// least one wave of such tiles (launch_gemm_simt picks it by sgemm128_fits).
bool sgemm128_fits(const Gemm &g);
int launch_sgemm128(const Gemm &g, cudaStream_t s);
// Triangular solve on device operands (t.A, t.B device pointers): recursive
// halving into device_gemm updates (native or emulated by the precision
// mode) and a substitution kernel for blocks of <= 64 rows. Sets *emulated
// when any update took the emulated path.
int trsm_device(const Trsm &t, cudaStream_t s, bool *emulated);
// The largest update GEMM trsm_device issues for t (its scratch bounds the
// solve's), or a Gemm with K == 0 when the triangle is a single leaf.
Gemm trsm_top_update(const Trsm &t);
// Parts of a solve or multiply, for pipelines that work through the order in
// blocks. trsm_solve_part solves rows (left) or columns (right) [lo, hi)
// whose right-hand sides are scale * B, against their diagonal block;
// trsm_update_part applies B[tgt] = scale B[tgt] - op(A)[tgt, src] X[src] (or
// the right-side mirror B[:, tgt] = scale B[:, tgt] - X[:, src] op(A)[src, tgt]).
// Blocks solved in substitution order, each after the update from those
// before it, give trsm_device. tri_forward: that order is ascending (the
// system matrix, op(A) for a left solve and op(A)^T for a right one, is
// lower); every update then reads op(A) inside the stored triangle.
bool tri_forward(const Trsm &t);
// The update of block tgt from block src as a GEMM on t's operands (alpha
// t.alpha, beta 1): sizes the scratch of a block pipeline.
Gemm tri_update_gemm(const Trsm &t, int64_t tgt_lo, int64_t tgt_hi, int64_t src_lo, int64_t src_hi);
// TRMM (a Trsm describes it: B = alpha op(A) B or alpha B op(A), in place):
// recursive halving into GEMM updates plus leaves of at most 256 rows that
// multiply by their completed diagonal block on the native kernels. Its
// scratch: one diagonal block and one leaf's vectors.
struct TrmmScratch {
    void *diag = nullptr, *temp = nullptr;
    int64_t ldt = 0;
    size_t diag_bytes = 0, temp_bytes = 0;
};
TrmmScratch trmm_scratch_sizes(const Trsm &t);
int trmm_device(const Trsm &t, const TrmmScratch &w, cudaStream_t s, bool *emulated);
// Parts of an out-of-place multiply into dst, a device buffer with B's
// layout; B is left unchanged. trmm_part_into writes rows (left) or columns
// (right) [lo, hi) of dst: alpha times their diagonal block times B's (its
// leaves multiply straight from B, without the staging copy of the in-place
// form). trmm_update_into adds alpha op(A)[tgt, src] B[src] (or B[:, src]
// op(A)[src, tgt]) to block tgt of dst. Every block's product, followed by
// the update from the blocks before it in substitution order, gives
// trmm_device's result.
int trmm_part_into(const Trsm &t, void *dst, int64_t lo, int64_t hi, const TrmmScratch &w, cudaStream_t s,
                   bool *emulated);
int trmm_update_into(const Trsm &t, void *dst, int64_t tgt_lo, int64_t tgt_hi, int64_t src_lo, int64_t src_hi,
                     cudaStream_t s, bool *emulated);
Gemm trmm_top_update(const Trsm &t);
int trsm_solve_part(const Trsm &t, int64_t lo, int64_t hi, cplx scale, cudaStream_t s, bool *emulated);
int trsm_update_part(const Trsm &t, int64_t tgt_lo, int64_t tgt_hi, int64_t src_lo, int64_t src_hi, cplx scale,
                     cudaStream_t s, bool *emulated);

}  // namespace bx
