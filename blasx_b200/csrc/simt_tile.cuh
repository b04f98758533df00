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

// ---- FP32 on the CUDA cores, 128 x 128 C tile per CTA of 256 threads ----------
//
// The 64 x 64 tile above computes 4 x 4 outputs per thread and loads one
// shared-memory value per FMA, which holds FP32 near 30% of the pipe. Here
// each thread reads two float4 of A and two of B per k (an 8 x 8 outer
// product: 64 FMAs for 4 loads), A and B stage through a double-buffered
// shared tile (one barrier per 8-deep k-tile, the next k-tile's global loads
// in flight during the current one's FMAs), and the epilogue loads two
// columns of a thread's C block before storing them. Same semantics: any
// transposes (ConjTrans is Trans for real data), ragged edges, C not read
// when beta == 0, the triangular-output mask.
namespace sg {
constexpr int TM = 128, TN = 128, TK = 8, THR = 256;
constexpr int PAD = 4;  // shared rows of 132 floats: 16-byte aligned float4 reads, conflict-free transposed stores
constexpr int LD_PER = TM * TK / THR;  // global elements of A (and of B) per thread per k-tile
static_assert(LD_PER * THR == TM * TK && TM == TN, "load mapping");

__device__ __forceinline__ bool tri_out(int uplo, int64_t diag, int64_t r, int64_t c) {
    return uplo && (uplo == 1 ? r - c > diag : r - c < diag);
}
}  // namespace sg
using namespace sg;

// Shared memory of one 128 x 128 tile: the double-buffered A and B k-tiles.
constexpr size_t sgemm128_smem_bytes() { return size_t(2) * 2 * TK * (TM + PAD) * sizeof(float); }

// C tile (bm, bn) of p (128 x 128); smem holds sgemm128_smem_bytes() bytes,
// 16-byte aligned.
__device__ __forceinline__ void sgemm128_tile(const SimtParams<float> &p, int64_t bm, int64_t bn, float *smem) {
    float (*As)[TK][TM + PAD] = reinterpret_cast<float (*)[TK][TM + PAD]>(smem);
    float (*Bs)[TK][TN + PAD] = reinterpret_cast<float (*)[TK][TN + PAD]>(smem + 2 * TK * (TM + PAD));
    const int ta = p.ta, tb = p.tb, M = p.M, N = p.N, K = p.K;
    const float alpha = p.alpha, beta = p.beta;
    const float *__restrict__ A = p.A;
    const float *__restrict__ B = p.B;
    float *__restrict__ C = p.C;
    const int64_t lda = p.lda, ldb = p.ldb, ldc = p.ldc;
    const int beta_zero = p.beta_zero, uplo = p.uplo;
    const int64_t diag = p.diag;
    const int tid = threadIdx.x;
    const int64_t m0 = bm * TM, n0 = bn * TN;
    // triangular output: a tile with no entry inside computes nothing
    if (uplo == 1 && m0 - (n0 + TN - 1) > diag) return;
    if (uplo == 2 && (m0 + TM - 1) - n0 < diag) return;
    const bool at = ta != NoTrans, bt = tb != NoTrans;

    // Element q (0 <= q < LD_PER) of this thread's share of a k-tile sits at
    // (row, k) = (r0 + q dr, k0 + q dk) of op(A) and (k, col) of op(B), with
    // consecutive threads along the operand's contiguous direction; its
    // global address is base + q * qstride, advanced by kstride per k-tile,
    // and its shared-memory slot is soff + q * sstride (all loop-invariant).
    struct Share {
        const float *ptr;
        int64_t qstride, kstride;
        int r, dr, k, dk, soff, sstride;
    };
    auto share = [&](const float *X, int64_t ld, bool tr, int64_t x0, int R) {
        Share d;
        // tr: the operand's k index is contiguous in memory (stored K x R); else its row / column index is
        d.r = tr ? tid / TK : tid % R;
        d.k = tr ? tid % TK : tid / R;
        d.dr = tr ? THR / TK : 0;
        d.dk = tr ? 0 : THR / R;
        d.ptr = tr ? X + d.k + (x0 + d.r) * ld : X + (x0 + d.r) + d.k * ld;
        d.qstride = tr ? int64_t(d.dr) * ld : int64_t(d.dk) * ld;
        d.kstride = tr ? TK : int64_t(TK) * ld;
        d.soff = d.k * (R + PAD) + d.r;
        d.sstride = d.dk * (R + PAD) + d.dr;
        return d;
    };
    // op(A) is M x K (row index m contiguous unless transposed); op(B) is K x N, stored K x N
    // (k contiguous) unless transposed
    Share sa = share(A, lda, at, m0, TM);
    Share sb = share(B, ldb, !bt, n0, TN);
    float ra[LD_PER], rb[LD_PER];
    auto load = [&](int64_t k0) {
#pragma unroll
        for (int q = 0; q < LD_PER; ++q) {
            const bool a_in = m0 + sa.r + q * sa.dr < M && k0 + sa.k + q * sa.dk < K;
            ra[q] = a_in ? sa.ptr[q * sa.qstride] : 0.f;
            const bool b_in = n0 + sb.r + q * sb.dr < N && k0 + sb.k + q * sb.dk < K;
            rb[q] = b_in ? sb.ptr[q * sb.qstride] : 0.f;
        }
        sa.ptr += sa.kstride;
        sb.ptr += sb.kstride;
    };
    auto store = [&](int buf) {
        float *as = &As[buf][0][0], *bs = &Bs[buf][0][0];
#pragma unroll
        for (int q = 0; q < LD_PER; ++q) {
            as[sa.soff + q * sa.sstride] = ra[q];
            bs[sb.soff + q * sb.sstride] = rb[q];
        }
    };

    // thread (tx, ty) owns rows ty*4 + {0..3}, 64 + ty*4 + {0..3} and columns tx*4 + {0..3}, 64 + tx*4 + {0..3}
    const int tx = tid % 16, ty = tid / 16;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    load(0);
    store(0);
    __syncthreads();
    for (int64_t k0 = 0, t = 0; k0 < K; k0 += TK, ++t) {
        const int cur = int(t & 1);
        const bool more = k0 + TK < K;
        if (more) load(k0 + TK);
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[cur][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[cur][kk][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[cur][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[cur][kk][64 + tx * 4]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        // the other buffer was last read before the previous barrier
        if (more) store(cur ^ 1);
        __syncthreads();
    }

    // epilogue: C = alpha acc + beta C; per pair of columns, all C loads before the stores
#pragma unroll
    for (int jp = 0; jp < 8; jp += 2) {
        float cin[2][8];
#pragma unroll
        for (int d = 0; d < 2; ++d)
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int j = jp + d;
                const int64_t gm = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
                const int64_t gn = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
                const bool in = !beta_zero && gm < M && gn < N && !tri_out(uplo, diag, gm, gn);
                cin[d][i] = in ? C[gm + gn * ldc] : 0.f;
            }
#pragma unroll
        for (int d = 0; d < 2; ++d)
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int j = jp + d;
                const int64_t gm = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
                const int64_t gn = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
                if (gm >= M || gn >= N || tri_out(uplo, diag, gm, gn)) continue;
                const float v = alpha * acc[i][j];
                C[gm + gn * ldc] = beta_zero ? v : fmaf(beta, cin[d][i], v);
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
