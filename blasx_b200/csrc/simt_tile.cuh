// simt_tile.cuh -- the portable SIMT GEMM tile (any dtype, any transpose,
// ragged edges, BLAS alpha / beta semantics: C not read when beta == 0), as
// device code shared by the standalone kernel (kernels_simt.cu) and the
// serving executor (executor.cu). One CTA of kSimtThreads threads computes a
// 64 x 64 C tile; each thread a 4 x 4 block of it, over 16-deep k steps
// staged in shared memory.
#pragma once

#include <cstdint>

#include "arith.cuh"
#include "runtime.h"

namespace bx {
namespace dev {

constexpr int kSimtBM = 64, kSimtBN = 64, kSimtBK = 16, kSimtThreads = 256;

template <typename T> struct SimtParams {
    int ta, tb, M, N, K;
    T alpha, beta;
    const T *A;
    int64_t lda;
    const T *B;
    int64_t ldb;
    T *C;
    int64_t ldc;
    int beta_zero;
    int uplo;  // triangular output: 0 all, 1 row - col <= diag, 2 row - col >= diag
    int64_t diag;
};

// Shared memory of one tile: the A and B k-steps.
template <typename T> constexpr size_t simt_smem_bytes() {
    return size_t(2) * kSimtBK * (kSimtBM + 1) * sizeof(T);
}

// C tile (bm, bn) of p; smem holds simt_smem_bytes<T>() bytes.
template <typename T>
__device__ __forceinline__ void simt_tile(const SimtParams<T> &p, int64_t bm, int64_t bn, T *smem) {
    using Ar = Arith<T>;
    constexpr int BM = kSimtBM, BN = kSimtBN, BK = kSimtBK, NT = kSimtThreads;
    T (*As)[BM + 1] = reinterpret_cast<T (*)[BM + 1]>(smem);
    T (*Bs)[BN + 1] = reinterpret_cast<T (*)[BN + 1]>(smem + BK * (BM + 1));
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int64_t m0 = bm * BM, n0 = bn * BN;
    const int ta = p.ta, tb = p.tb, M = p.M, N = p.N, K = p.K;
    const T *__restrict__ A = p.A;
    const T *__restrict__ B = p.B;
    // triangular output: a tile with no entry inside computes nothing
    if (p.uplo == 1 && m0 - (n0 + BN - 1) > p.diag) return;
    if (p.uplo == 2 && (m0 + BM - 1) - n0 < p.diag) return;
    T acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = Ar::zero();

    for (int64_t k0 = 0; k0 < K; k0 += BK) {
        for (int e = tid; e < BM * BK; e += NT) {
            int mm, kk;
            if (ta == NoTrans) { mm = e % BM; kk = e / BM; }
            else { kk = e % BK; mm = e / BK; }
            const int64_t gm = m0 + mm, gk = k0 + kk;
            T v = Ar::zero();
            if (gm < M && gk < K) {
                v = ta == NoTrans ? A[gm + gk * p.lda] : A[gk + gm * p.lda];
                if (ta == ConjT) v = Ar::conj(v);
            }
            As[kk][mm] = v;
        }
        for (int e = tid; e < BN * BK; e += NT) {
            int nn, kk;
            if (tb == NoTrans) { kk = e % BK; nn = e / BK; }
            else { nn = e % BN; kk = e / BN; }
            const int64_t gn = n0 + nn, gk = k0 + kk;
            T v = Ar::zero();
            if (gn < N && gk < K) {
                v = tb == NoTrans ? B[gk + gn * p.ldb] : B[gn + gk * p.ldb];
                if (tb == ConjT) v = Ar::conj(v);
            }
            Bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = Ar::fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t gn = n0 + ty + 16 * j;
        if (gn >= N) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t gm = m0 + tx + 16 * i;
            if (gm >= M) continue;
            if (p.uplo && (p.uplo == 1 ? gm - gn > p.diag : gm - gn < p.diag)) continue;
            T *cp = &p.C[gm + gn * p.ldc];
            T v = Ar::mul(p.alpha, acc[i][j]);
            if (!p.beta_zero) v = Ar::add(v, Ar::mul(p.beta, *cp));
            *cp = v;
        }
    }
}

// beta-scaling of C (alpha == 0 or K == 0): entries t in [t0, t1) of the
// column-major M x N block, C not read when beta == 0.
template <typename T>
__device__ __forceinline__ void scale_range(int M, T beta, T *__restrict__ C, int64_t ldc, int beta_zero,
                                            int uplo, int64_t diag, int64_t t0, int64_t t1, int64_t stride) {
    using Ar = Arith<T>;
    for (int64_t t = t0; t < t1; t += stride) {
        const int64_t i = t % M, j = t / M;
        if (uplo && (uplo == 1 ? i - j > diag : i - j < diag)) continue;
        T *cp = &C[i + j * ldc];
        *cp = beta_zero ? Ar::zero() : Ar::mul(beta, *cp);
    }
}

}  // namespace dev
}  // namespace bx
