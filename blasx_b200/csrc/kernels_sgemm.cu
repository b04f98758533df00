// kernels_sgemm.cu -- FP32 GEMM on the CUDA cores for problems that fill the
// GPU: 128 x 128 C tile per CTA, 8 x 8 outputs per thread.
//
// The portable SIMT kernel (kernels_simt.cu) computes 4 x 4 outputs per
// thread and loads one shared-memory value per FMA, which holds FP32 near
// 30% of the pipe. Here each thread reads two float4 of A and two of B per k
// (an 8 x 8 outer product: 64 FMAs for 4 loads), A and B stage through a
// double-buffered shared tile (one barrier per 8-deep k-tile, the next
// k-tile's global loads in flight during the current one's FMAs), and the
// epilogue loads two columns of a thread's C block before storing them.
// Same semantics as the SIMT kernel: any transposes (ConjTrans is Trans for
// real data), ragged edges, C not read when beta == 0, the triangular-output
// mask and the emulated path's guard.
#include "kernels.h"

namespace bx {
namespace {

constexpr int TM = 128, TN = 128, TK = 8, THR = 256;
constexpr int PAD = 4;  // shared rows of 132 floats: 16-byte aligned float4 reads, conflict-free transposed stores
constexpr int LD_PER = TM * TK / THR;  // global elements of A (and of B) per thread per k-tile
static_assert(LD_PER * THR == TM * TK && TM == TN, "load mapping");

__device__ __forceinline__ bool tri_out(int uplo, int64_t diag, int64_t r, int64_t c) {
    return uplo && (uplo == 1 ? r - c > diag : r - c < diag);
}

__global__ void __launch_bounds__(THR, 2)
    sgemm128_kernel(int ta, int tb, int M, int N, int K, float alpha, const float *__restrict__ A, int64_t lda,
                    const float *__restrict__ B, int64_t ldb, float beta, float *__restrict__ C, int64_t ldc,
                    int beta_zero, const int *guard, int uplo, int64_t diag) {
    if (guard && *guard != 0) return;  // the emulated path produced C
    __shared__ __align__(16) float As[2][TK][TM + PAD];
    __shared__ __align__(16) float Bs[2][TK][TN + PAD];
    const int tid = threadIdx.x;
    const int64_t m0 = int64_t(blockIdx.x) * TM, n0 = int64_t(blockIdx.y) * TN;
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

}  // namespace

bool sgemm128_fits(const Gemm &g) {
    const int64_t tiles = ((g.M + TM - 1) / TM) * ((g.N + TN - 1) / TN);
    return g.dt == DType::F32 && tiles >= 148 && g.M <= INT32_MAX && g.N <= INT32_MAX && g.K <= INT32_MAX &&
           (g.N + TN - 1) / TN <= 65535;
}

int launch_sgemm128(const Gemm &g, cudaStream_t s) {
    dim3 grid(unsigned((g.M + TM - 1) / TM), unsigned((g.N + TN - 1) / TN));
    sgemm128_kernel<<<grid, THR, 0, s>>>(g.ta, g.tb, int(g.M), int(g.N), int(g.K), float(g.alpha.re),
                                          static_cast<const float *>(g.A), g.lda, static_cast<const float *>(g.B),
                                          g.ldb, float(g.beta.re), static_cast<float *>(g.C), g.ldc,
                                          g.beta_zero() ? 1 : 0, g.guard, g.uplo, g.diag);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

}  // namespace bx
