// kernels_simt.cu -- portable SIMT GEMM kernel, the beta-scale kernel and the
// scaled-add kernel of the host pipeline.
//
// The SIMT kernel is the correctness baseline of the device path: any dtype,
// any transpose, ragged edges, BLAS alpha/beta semantics (C not read when
// beta == 0). Fast paths live in kernels_dmma.cu (FP64 pipe) and the Ozaki
// INT8 tensor-core path.
#include <algorithm>

#include "arith.cuh"
#include "kernels.h"
#include "simt_tile.cuh"

namespace bx {

namespace {

using namespace dev;

constexpr int BM = kSimtBM, BN = kSimtBN, NT = kSimtThreads;

template <typename T>
__global__ void __launch_bounds__(NT) gemm_simt_kernel(const SimtParams<T> p, const int *guard) {
    if (guard && *guard != 0) return;  // the emulated path produced C
    __shared__ T smem[2 * kSimtBK * (kSimtBM + 1)];
    simt_tile<T>(p, blockIdx.x, blockIdx.y, smem);
}

template <typename T>
__global__ void scale_kernel(int M, int N, T beta, T *__restrict__ C, int64_t ldc, int beta_zero,
                             int uplo, int64_t diag) {
    scale_range<T>(M, beta, C, ldc, beta_zero, uplo, diag, blockIdx.x * int64_t(blockDim.x) + threadIdx.x,
                   int64_t(M) * N, int64_t(gridDim.x) * blockDim.x);
}

// C(i, j) += beta X(i, j): blockIdx.y strides over columns, threads over rows.
template <typename T>
__global__ void add_scaled_kernel(int M, int N, T beta, const T *__restrict__ X, int64_t ldx,
                                  T *__restrict__ C, int64_t ldc, int uplo, int64_t diag) {
    using Ar = Arith<T>;
    for (int64_t j = blockIdx.y; j < N; j += gridDim.y)
        for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < M;
             i += int64_t(gridDim.x) * blockDim.x) {
            if (uplo && (uplo == 1 ? i - j > diag : i - j < diag)) continue;
            T *cp = &C[i + j * ldc];
            *cp = Ar::add(*cp, Ar::mul(beta, X[i + j * ldx]));
        }
}

template <typename T> int launch_add_scaled_t(const Gemm &g, const void *X, int64_t ldx, cudaStream_t s) {
    dim3 grid(unsigned(std::min<int64_t>(8, (g.M + 255) / 256)), unsigned(std::min<int64_t>(g.N, 65535)));
    add_scaled_kernel<T><<<grid, 256, 0, s>>>(int(g.M), int(g.N), from_cplx<T>(g.beta),
                                              static_cast<const T *>(X), ldx, static_cast<T *>(g.C), g.ldc,
                                              g.uplo, g.diag);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

// One CTA of 32 x 8 threads per 32 x 32 tile of X that holds entries to
// complete (the other triangle and the diagonal). A mirrored tile is read
// from the stored triangle with coalesced column reads into shared memory and
// written back transposed, again column by column; a diagonal tile reads
// itself whole before writing only its other triangle.
constexpr int kCompTile = 32, kCompRows = 8;

template <typename T>
__global__ void __launch_bounds__(kCompTile * kCompRows)
complete_operand_kernel(int form, T *__restrict__ X, int64_t ldx, int n) {
    using Ar = Arith<T>;
    const bool upper = form == kSymUpper || form == kHermUpper || form == kTriUpper || form == kTriUpperUnit;
    const bool herm = form == kHermUpper || form == kHermLower;
    const bool tri = form >= kTriUpper;
    const bool unit = form == kTriUpperUnit || form == kTriLowerUnit;
    // target tile: rows r0.., columns c0..; with the upper triangle stored the
    // targets lie on or below the diagonal (tile row >= tile column)
    const int tr = blockIdx.x, tc = blockIdx.y;
    if (upper ? tr < tc : tr > tc) return;
    const int64_t r0 = int64_t(tr) * kCompTile, c0 = int64_t(tc) * kCompTile;
    const int tx = threadIdx.x, ty = threadIdx.y;
    __shared__ T sm[kCompTile][kCompTile + 1];  // sm[i - r0][j - c0] = X(j, i)
    if (!tri) {
#pragma unroll
        for (int k = 0; k < kCompTile; k += kCompRows) {
            const int64_t j = c0 + tx, i = r0 + ty + k;  // source X(j, i): column i
            if (j < n && i < n) sm[ty + k][tx] = X[j + i * ldx];
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < kCompTile; k += kCompRows) {
        const int64_t i = r0 + tx, j = c0 + ty + k;  // target X(i, j): column j
        if (i >= n || j >= n) continue;
        T *xp = &X[i + j * ldx];
        if (i == j) {
            if (unit) *xp = Ar::one();
            else if (herm) *xp = Ar::real_part(*xp);
            continue;
        }
        if (upper ? i < j : i > j) continue;  // stored
        if (tri) *xp = Ar::zero();
        else *xp = herm ? Ar::conj(sm[tx][ty + k]) : sm[tx][ty + k];
    }
}

template <typename T> int launch_complete_t(int form, void *X, int64_t ldx, int64_t n, cudaStream_t s) {
    const int64_t tiles = (n + kCompTile - 1) / kCompTile;
    if (tiles > 65535) return set_error(BLASX_ERR_UNSUPPORTED, "operand order too large to complete");
    complete_operand_kernel<T><<<dim3(unsigned(tiles), unsigned(tiles)), dim3(kCompTile, kCompRows), 0, s>>>(
        form, static_cast<T *>(X), ldx, int(n));
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

template <typename T> int launch_simt_t(const Gemm &g, cudaStream_t s) {
    dim3 grid(unsigned((g.M + BM - 1) / BM), unsigned((g.N + BN - 1) / BN));
    if (grid.y > 65535) return set_error(BLASX_ERR_UNSUPPORTED, "N too large for SIMT grid");
    const SimtParams<T> p{g.ta, g.tb, int(g.M), int(g.N), int(g.K), from_cplx<T>(g.alpha),
                          from_cplx<T>(g.beta), static_cast<const T *>(g.A), g.lda,
                          static_cast<const T *>(g.B), g.ldb, static_cast<T *>(g.C), g.ldc,
                          g.beta_zero() ? 1 : 0, g.uplo, g.diag};
    gemm_simt_kernel<T><<<grid, NT, 0, s>>>(p, g.guard);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

template <typename T> int launch_scale_t(const Gemm &g, cudaStream_t s) {
    const int64_t total = g.M * g.N;
    int blocks = int((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    scale_kernel<T><<<blocks, 256, 0, s>>>(int(g.M), int(g.N), from_cplx<T>(g.beta),
                                            static_cast<T *>(g.C), g.ldc, g.beta_zero() ? 1 : 0, g.uplo,
                                            g.diag);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

}  // namespace

int launch_gemm_simt(const Gemm &g, cudaStream_t s) {
    switch (g.dt) {
        case DType::F32: return sgemm128_fits(g) ? launch_sgemm128(g, s) : launch_simt_t<float>(g, s);
        case DType::F64: return launch_simt_t<double>(g, s);
        case DType::C64: return launch_simt_t<c2>(g, s);
        default: return launch_simt_t<z2>(g, s);
    }
}

int launch_complete_operand(DType dt, int form, void *X, int64_t ldx, int64_t n, cudaStream_t s) {
    if (form == kGeneral || n <= 0) return BLASX_OK;
    switch (dt) {
        case DType::F32: return launch_complete_t<float>(form, X, ldx, n, s);
        case DType::F64: return launch_complete_t<double>(form, X, ldx, n, s);
        case DType::C64: return launch_complete_t<c2>(form, X, ldx, n, s);
        default: return launch_complete_t<z2>(form, X, ldx, n, s);
    }
}

// One thread per diagonal entry: (r, r - off) for r in the block.
template <typename R>
__global__ void real_diagonal_kernel(R *C, int64_t ldc, int64_t m, int64_t n, int64_t off) {
    const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    const int64_t r = (off > 0 ? off : 0) + t, c = r - off;
    if (r < m && c >= 0 && c < n) C[2 * (r + c * ldc) + 1] = R(0);
}

int launch_real_diagonal(DType dt, void *C, int64_t ldc, int64_t m, int64_t n, int64_t off, cudaStream_t s) {
    if (!is_complex(dt) || m <= 0 || n <= 0) return BLASX_OK;
    const int64_t len = std::min(m - std::max<int64_t>(off, 0), n + std::min<int64_t>(off, 0));
    if (len <= 0) return BLASX_OK;
    const unsigned blocks = unsigned((len + 255) / 256);
    if (dt == DType::C128)
        real_diagonal_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double *>(C), ldc, m, n, off);
    else
        real_diagonal_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float *>(C), ldc, m, n, off);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

int launch_add_scaled(const Gemm &g, const void *X, int64_t ldx, cudaStream_t s) {
    if (g.M == 0 || g.N == 0 || g.beta_zero()) return BLASX_OK;
    switch (g.dt) {
        case DType::F32: return launch_add_scaled_t<float>(g, X, ldx, s);
        case DType::F64: return launch_add_scaled_t<double>(g, X, ldx, s);
        case DType::C64: return launch_add_scaled_t<c2>(g, X, ldx, s);
        default: return launch_add_scaled_t<z2>(g, X, ldx, s);
    }
}

int launch_scale(const Gemm &g, cudaStream_t s) {
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    switch (g.dt) {
        case DType::F32: return launch_scale_t<float>(g, s);
        case DType::F64: return launch_scale_t<double>(g, s);
        case DType::C64: return launch_scale_t<c2>(g, s);
        default: return launch_scale_t<z2>(g, s);
    }
}

}  // namespace bx
