// dmma_tile.cuh -- the native FP64 / complex128 GEMM tile on the FP64 tensor
// pipe (DMMA), as device code shared by the standalone kernels
// (kernels_dmma.cu) and the serving executor (executor.cu).
//
// One CTA of Tile<CPLX, G>::THREADS threads computes one C tile:
//   * 8 warps in a 2 x 4 grid (FP64 128x128 tile, complex128 64x128), or 4
//     warps in a 2 x 2 grid (FP64 64x64 tile, G = 1); a warp owns a block of
//     accumulators in registers;
//   * operand tiles are staged global -> shared through a 3-stage cp.async
//     ring. Each operand keeps the contiguity it has in global memory: a
//     k-contiguous source (A transposed, B not) lands as [m][k] rows padded
//     by 4 doubles, an m/n-contiguous source as [k][m] rows padded by 4, so
//     every copy is a 16-byte cp.async along the contiguous direction and
//     every fragment load (8 rows x 4 doubles or 4 rows x 8 doubles) falls on
//     disjoint bank groups;
//   * ragged edges: the src-size operand of cp.async zero-fills the part of
//     a chunk beyond M, N or K, so nothing outside the matrices is read;
//   * the epilogue applies alpha / beta in FP64 and never reads C when
//     beta == 0 (BLAS semantics).
// Complex128 keeps real and imaginary planes separately in shared memory and
// issues four real DMMAs per fragment pair (re += ar br - ai bi,
// im += ar bi + ai br); conjugation flips the sign of the imaginary fragment.
#pragma once

#include <cstdint>

#include "runtime.h"

namespace bx {
namespace dev {

// CTA geometry. G selects the FP64 variant: 0 = a 128x128 C tile, 8 warps
// (2 x 4) of 64x32 accumulators each; 1 = a 64x64 C tile, 4 warps (2 x 2) of
// 32x32, two CTAs per SM, for problems with too few 128x128 tiles to occupy
// every SM (one CTA computes its whole K extent, at one SM's FP64 rate).
template <bool CPLX, int G = 0> struct Tile;
template <> struct Tile<false, 0> {
    static constexpr int THREADS = 256, WARPS_N = 4;
    static constexpr int BM = 128, BN = 128, MT = 4, NT = 4, BK = 32, STAGES = 3;
};
template <> struct Tile<false, 1> {
    static constexpr int THREADS = 128, WARPS_N = 2;
    static constexpr int BM = 64, BN = 64, MT = 2, NT = 4, BK = 32, STAGES = 3;
};
template <> struct Tile<true, 0> {
    static constexpr int THREADS = 256, WARPS_N = 4;
    static constexpr int BM = 64, BN = 128, MT = 2, NT = 4, BK = 16, STAGES = 3;
};

// Shared-memory geometry of one operand tile (rows x k) for a given source
// contiguity. KC: [row][k] with stride BK+4; else [k][row] with stride R+4.
// A 64-bit shared load is served per half-warp (lanes g < 4 or g >= 4, all
// t): with a stride of 4 (mod 16 doubles) the 16 lanes of a fragment load,
// at stride*t + g or stride*g + t, fall on 16 distinct bank pairs.
template <int R, int BK, bool KC> struct SmemOp {
    static constexpr int stride = KC ? BK + 4 : R + 4;
    static_assert(stride % 16 == 4, "bank-conflict-free fragment loads");
    static constexpr int plane = KC ? R * stride : BK * stride;  // doubles
    __device__ static int idx(int r, int k) { return KC ? r * stride + k : k * stride + r; }
};

struct DmmaParams {
    int M, N, K, ta, tb;
    const double *A;
    int64_t lda;
    const double *B;
    int64_t ldb;
    double *C;
    int64_t ldc;
    double alpha_re, alpha_im, beta_re, beta_im;
    int beta_zero;
    int tiles_m, tiles_n;
    int vec_a, vec_b;  // 16-byte copies allowed (ld even, base 16-byte aligned)
    const int *guard;  // when set, run only if *guard == 0
    int uplo;          // triangular output: 0 all, 1 row - col <= diag, 2 row - col >= diag
    int64_t diag;
};

__device__ __forceinline__ bool tri_keep(int uplo, int64_t diag, int64_t r, int64_t c) {
    return uplo == 0 || (uplo == 1 ? r - c <= diag : r - c >= diag);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// cp.async of `bytes` (8 or 16) with `src_bytes` valid bytes; the rest of the
// destination is zero-filled and no memory past src_bytes is read.
template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void *src, int src_bytes) {
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                     "r"(src_bytes)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                     "r"(src_bytes)
                     : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// D(16x8) += A(16xKI, row) * B(KIx8, col), f64. Fragments (g = lane/4,
// t = lane%4, q < KI/4, h < 2): a[2q+h] = A[g+8h][t+4q], b[q] = B[t+4q][g];
// c0,c1 = C[g][2t..2t+1], c2,c3 = C[g+8][2t..2t+1].
template <int KI> struct Dmma;
template <> struct Dmma<4> {
    __device__ static void run(double (&c)[4], const double *a, const double *b) {
        asm volatile(
            "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(b[0]));
    }
};
template <> struct Dmma<8> {
    __device__ static void run(double (&c)[4], const double *a, const double *b) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
    }
};
template <> struct Dmma<16> {
    __device__ static void run(double (&c)[4], const double *a, const double *b) {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
            "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
            : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]),
              "d"(a[7]), "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
    }
};

// Copies the R x BK operand tile at (r0, k0) of a column-major source into
// shared memory. KC: the source is k-contiguous (element (r, k) at
// src[k + r*ld]); else r-contiguous (src[r + k*ld]). V doubles per copy.
template <int R, int BK, bool KC, bool CPLX, int V, int THREADS>
__device__ __forceinline__ void load_tile(uint32_t sbase, const double *src, int64_t ld,
                                          int r0, int k0, int rows, int kdim, int tid) {
    using S = SmemOp<R, BK, KC>;
    constexpr int CHUNKS = R * BK / V;
    static_assert(CHUNKS % THREADS == 0, "tile / thread mismatch");
    constexpr int PER_ROW = KC ? BK / V : R / V;  // chunks along the contiguous dim
#pragma unroll
    for (int i = 0; i < CHUNKS / THREADS; ++i) {
        const int e = tid + i * THREADS;
        const int c = (e % PER_ROW) * V, o = e / PER_ROW;  // contiguous / other coordinate
        const int r = KC ? o : c, k = KC ? c : o;
        const int gr = r0 + r, gk = k0 + k;
        int valid;  // elements of this chunk inside the matrix
        if (KC) valid = (gr < rows) ? min(V, kdim - gk) : 0;
        else valid = (gk < kdim) ? min(V, rows - gr) : 0;
        valid = max(valid, 0);
        const int64_t off = valid ? (KC ? gk + int64_t(gr) * ld : gr + int64_t(gk) * ld) : 0;
        const uint32_t dst = sbase + uint32_t(S::idx(r, k)) * 8u;
        if (!CPLX) {
            cp_async<V * 8>(dst, src + off, valid * 8);
        } else {  // complex element = (re, im): split into the two planes
            const double *p = src + 2 * off;
            cp_async<8>(dst, p, valid * 8);
            cp_async<8>(dst + uint32_t(S::plane) * 8u, p + 1, valid * 8);
        }
    }
}

// One C tile of one problem (`tile` in the grouped raster order below).
template <bool CPLX, bool AKC, bool BKC, int KI, int G = 0>
__device__ __forceinline__ void dmma_tile(const DmmaParams &p, const int tile, double *smem) {
    using TL = Tile<CPLX, G>;
    constexpr int T = TL::THREADS;
    constexpr int BM = TL::BM, BN = TL::BN, MT = TL::MT, NT = TL::NT, BK = TL::BK;
    constexpr int STAGES = TL::STAGES;
    using SA = SmemOp<BM, BK, AKC>;
    using SB = SmemOp<BN, BK, BKC>;
    constexpr int PLANES = CPLX ? 2 : 1;
    constexpr int A_STAGE = PLANES * SA::plane, B_STAGE = PLANES * SB::plane;  // doubles
    constexpr int IM = CPLX ? 1 : 0;

    double *sA = smem;
    double *sB = smem + STAGES * A_STAGE;

    // grouped rasterisation: 8 tile-rows per group keeps A panels hot in L2
    constexpr int GROUP = 8;
    const int per_group = GROUP * p.tiles_n;
    const int group = tile / per_group;
    const int first_m = group * GROUP;
    const int gsize = min(p.tiles_m - first_m, GROUP);
    const int tm = first_m + (tile % per_group) % gsize;
    const int tn = (tile % per_group) / gsize;
    const int m0 = tm * BM, n0 = tn * BN;
    // triangular output: a tile with no entry inside computes nothing (uniform per CTA)
    if (p.uplo == 1 && int64_t(m0) - (n0 + BN - 1) > p.diag) return;
    if (p.uplo == 2 && int64_t(m0 + BM - 1) - n0 < p.diag) return;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp / TL::WARPS_N, wn = warp % TL::WARPS_N;
    const int g = lane >> 2, t = lane & 3;

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kt * BK;
        const uint32_t a_base = smem_u32(sA + stage * A_STAGE);
        const uint32_t b_base = smem_u32(sB + stage * B_STAGE);
        if (!CPLX && p.vec_a)
            load_tile<BM, BK, AKC, CPLX, 2, T>(a_base, p.A, p.lda, m0, k0, p.M, p.K, tid);
        else
            load_tile<BM, BK, AKC, CPLX, 1, T>(a_base, p.A, p.lda, m0, k0, p.M, p.K, tid);
        if (!CPLX && p.vec_b)
            load_tile<BN, BK, BKC, CPLX, 2, T>(b_base, p.B, p.ldb, n0, k0, p.N, p.K, tid);
        else
            load_tile<BN, BK, BKC, CPLX, 1, T>(b_base, p.B, p.ldb, n0, k0, p.N, p.K, tid);
    };

    double acc[PLANES][MT][NT][4];
#pragma unroll
    for (int pl = 0; pl < PLANES; ++pl)
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int r = 0; r < 4; ++r) acc[pl][i][j][r] = 0.0;

    const int ktiles = (p.K + BK - 1) / BK;
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < ktiles) load_stage(s, s);
        cp_async_commit();
    }

    // sign applied to the imaginary fragments: conj(A) / conj(B)
    const double sa = (CPLX && p.ta == ConjT) ? -1.0 : 1.0;
    const double sb = (CPLX && p.tb == ConjT) ? -1.0 : 1.0;
    const int arow = wm * (MT * 16) + g, bcol = wn * (NT * 8) + g;

    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nk = kt + STAGES - 1;
            if (nk < ktiles) load_stage(nk % STAGES, nk);
            cp_async_commit();
        }
        const double *a_s = sA + (kt % STAGES) * A_STAGE;
        const double *b_s = sB + (kt % STAGES) * B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BK; kk += KI) {
            double bf[PLANES][NT][KI / 4];
#pragma unroll
            for (int pl = 0; pl < PLANES; ++pl)
#pragma unroll
                for (int j = 0; j < NT; ++j)
#pragma unroll
                    for (int q = 0; q < KI / 4; ++q)
                        bf[pl][j][q] = b_s[pl * SB::plane + SB::idx(bcol + j * 8, kk + t + 4 * q)];
            if (CPLX) {
#pragma unroll
                for (int j = 0; j < NT; ++j)
#pragma unroll
                    for (int q = 0; q < KI / 4; ++q) bf[IM][j][q] *= sb;
            }
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                double af[PLANES][KI / 2];
#pragma unroll
                for (int pl = 0; pl < PLANES; ++pl)
#pragma unroll
                    for (int q = 0; q < KI / 4; ++q)
#pragma unroll
                        for (int h = 0; h < 2; ++h)
                            af[pl][2 * q + h] =
                                a_s[pl * SA::plane + SA::idx(arow + i * 16 + 8 * h, kk + t + 4 * q)];
                if (!CPLX) {
#pragma unroll
                    for (int j = 0; j < NT; ++j) Dmma<KI>::run(acc[0][i][j], af[0], bf[0][j]);
                } else {
                    double an[KI / 2];  // -conj-adjusted imaginary part of A
#pragma unroll
                    for (int q = 0; q < KI / 2; ++q) {
                        af[IM][q] *= sa;
                        an[q] = -af[IM][q];
                    }
#pragma unroll
                    for (int j = 0; j < NT; ++j) {
                        Dmma<KI>::run(acc[0][i][j], af[0], bf[0][j]);
                        Dmma<KI>::run(acc[0][i][j], an, bf[IM][j]);
                        Dmma<KI>::run(acc[IM][i][j], af[0], bf[IM][j]);
                        Dmma<KI>::run(acc[IM][i][j], af[IM], bf[0][j]);
                    }
                }
            }
        }
    }
    cp_async_wait<0>();

    // epilogue: C = alpha acc + beta C (C unread when beta == 0). The C values
    // of one row block (NT x 4 per thread) are all loaded before any store of
    // that block, so their DRAM round trips overlap instead of alternating
    // with the stores.
    const int64_t es = CPLX ? 2 : 1;
#pragma unroll
    for (int i = 0; i < MT; ++i) {
        double cin[NT][4][PLANES];
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = m0 + wm * (MT * 16) + i * 16 + g + (r >= 2 ? 8 : 0);
                const int col = n0 + wn * (NT * 8) + j * 8 + 2 * t + (r & 1);
                const bool in = !p.beta_zero && row < p.M && col < p.N && tri_keep(p.uplo, p.diag, row, col);
                const double *cp = p.C + (row + int64_t(col) * p.ldc) * es;
#pragma unroll
                for (int pl = 0; pl < PLANES; ++pl) cin[j][r][pl] = in ? cp[pl] : 0.0;
            }
#pragma unroll
        for (int j = 0; j < NT; ++j) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = m0 + wm * (MT * 16) + i * 16 + g + (r >= 2 ? 8 : 0);
                const int col = n0 + wn * (NT * 8) + j * 8 + 2 * t + (r & 1);
                if (row >= p.M || col >= p.N || !tri_keep(p.uplo, p.diag, row, col)) continue;
                double *cp = p.C + (row + int64_t(col) * p.ldc) * es;
                if (!CPLX) {
                    double v = p.alpha_re * acc[0][i][j][r];
                    if (!p.beta_zero) v = fma(p.beta_re, cin[j][r][0], v);
                    *cp = v;
                } else {
                    const double xr = acc[0][i][j][r], xi = acc[IM][i][j][r];
                    double vr = p.alpha_re * xr - p.alpha_im * xi;
                    double vi = p.alpha_re * xi + p.alpha_im * xr;
                    if (!p.beta_zero) {
                        const double cr = cin[j][r][0], ci = cin[j][r][PLANES - 1];
                        vr += p.beta_re * cr - p.beta_im * ci;
                        vi += p.beta_re * ci + p.beta_im * cr;
                    }
                    cp[0] = vr;
                    cp[1] = vi;
                }
            }
        }
    }
}


// Shared-memory bytes of one C tile of the given layout.
template <bool CPLX, bool AKC, bool BKC, int G = 0> constexpr size_t dmma_smem_bytes() {
    using TL = Tile<CPLX, G>;
    return size_t(TL::STAGES) * (CPLX ? 2 : 1) *
           (SmemOp<TL::BM, TL::BK, AKC>::plane + SmemOp<TL::BN, TL::BK, BKC>::plane) * sizeof(double);
}

template <bool CPLX, int G = 0> DmmaParams make_params(const Gemm &g) {
    using TL = Tile<CPLX, G>;
    DmmaParams p;
    p.M = int(g.M); p.N = int(g.N); p.K = int(g.K);
    p.ta = g.ta; p.tb = g.tb;
    p.A = static_cast<const double *>(g.A); p.lda = g.lda;
    p.B = static_cast<const double *>(g.B); p.ldb = g.ldb;
    p.C = static_cast<double *>(g.C); p.ldc = g.ldc;
    p.alpha_re = g.alpha.re; p.alpha_im = g.alpha.im;
    p.beta_re = g.beta.re; p.beta_im = g.beta.im;
    p.beta_zero = g.beta_zero() ? 1 : 0;
    p.tiles_m = int((g.M + TL::BM - 1) / TL::BM);
    p.tiles_n = int((g.N + TL::BN - 1) / TL::BN);
    p.vec_a = (g.lda % 2 == 0) && (reinterpret_cast<uintptr_t>(g.A) % 16 == 0);
    p.vec_b = (g.ldb % 2 == 0) && (reinterpret_cast<uintptr_t>(g.B) % 16 == 0);
    p.guard = g.guard;
    p.uplo = g.uplo;
    p.diag = g.diag;
    return p;
}

}  // namespace dev
}  // namespace bx
