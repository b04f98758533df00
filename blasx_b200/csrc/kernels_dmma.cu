// kernels_dmma.cu -- native FP64 and complex128 GEMM on the FP64 tensor pipe.
//
// Replaces the per-tile cublasDgemm / cublasZgemm call of the reference
// (blas/blasx_dgemm.c:87-95, blas/blasx_zgemm.c:88) with a hand-written
// sm_100a kernel built on DMMA (mma.sync m16n8k{4,8,16}, f64 in, f64
// accumulate).
//
// The tile itself (DMMA fragments, the cp.async ring, the alpha / beta
// epilogue) is dmma_tile.cuh, shared with the serving executor; this file
// holds the launches: one CTA per C tile, with the CTA geometry chosen by
// the estimated SM utilisation.
#include <cstdint>
#include <cstdlib>

#include "dmma_tile.cuh"
#include "kernels.h"

namespace bx {

namespace {

using namespace dev;

template <bool CPLX, bool AKC, bool BKC, int KI, int G>
__global__ void __launch_bounds__(Tile<CPLX, G>::THREADS, 1) dmma_gemm_kernel(const DmmaParams p) {
    if (p.guard && *p.guard != 0) return;  // the emulated path produced C
    extern __shared__ __align__(16) double smem[];
    dmma_tile<CPLX, AKC, BKC, KI, G>(p, blockIdx.x, smem);
}

template <bool CPLX, bool AKC, bool BKC, int KI, int G>
int launch_cfg(const DmmaParams &p, cudaStream_t s) {
    using TL = Tile<CPLX, G>;
    constexpr int PLANES = CPLX ? 2 : 1;
    constexpr size_t smem = size_t(TL::STAGES) * PLANES *
                            (SmemOp<TL::BM, TL::BK, AKC>::plane + SmemOp<TL::BN, TL::BK, BKC>::plane) *
                            sizeof(double);
    static_assert(smem <= 227 * 1024, "shared memory budget");
    auto kern = dmma_gemm_kernel<CPLX, AKC, BKC, KI, G>;
    BX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int64_t tiles = int64_t(p.tiles_m) * p.tiles_n;
    kern<<<unsigned(tiles), TL::THREADS, smem, s>>>(p);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

// Instruction K of the FP64 MMA: 16 by default (BLASX_DMMA_K = 4, 8 or 16).
int dmma_k() {
    static const int k = [] {
        const char *e = getenv("BLASX_DMMA_K");
        const int v = e ? atoi(e) : 16;
        return (v == 4 || v == 8) ? v : 16;
    }();
    return k;
}

// FP64 CTA geometry, by the estimated fraction of the SMs' FP64 pipes kept
// busy: a grid of t CTAs, r resident per SM, runs in ceil(t / (r S)) waves,
// so the busy fraction is t / (ceil(t / (r S)) r S). The 128x128 tile runs
// one CTA per SM; the 64x64 tile two, at an assumed 85% of the larger
// tile's per-SM rate (more shared-memory traffic per flop). BLASX_DMMA_TILE
// = 64 or 128 forces one.
int dmma_geometry(int64_t M, int64_t N) {
    static const int forced = [] {
        const char *e = getenv("BLASX_DMMA_TILE");
        const int v = e ? atoi(e) : 0;
        return v == 64 ? 1 : (v == 128 ? 0 : -1);
    }();
    if (forced >= 0) return forced;
    static const int sms = [] {
        int dev = 0, n = 148;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            n = 148;
        return n;
    }();
    // share of the SM slots of all waves that hold useful output: occupancy
    // of the last wave times the part of each tile inside M x N
    auto useful = [&](int64_t edge, int per_sm) {
        const int64_t tiles = ((M + edge - 1) / edge) * ((N + edge - 1) / edge);
        const int64_t slots = int64_t(sms) * per_sm;
        const int64_t waves = (tiles + slots - 1) / slots;
        return double(M) * double(N) / (double(waves * slots) * double(edge * edge));
    };
    const double big = useful(128, 1);
    const double small = 0.85 * useful(64, 2);
    return small > big ? 1 : 0;
}

template <bool CPLX, bool AKC, bool BKC, int G> int launch_kg(const DmmaParams &p, cudaStream_t s) {
    switch (dmma_k()) {
        case 4: return launch_cfg<CPLX, AKC, BKC, 4, G>(p, s);
        case 8: return launch_cfg<CPLX, AKC, BKC, 8, G>(p, s);
        default: return launch_cfg<CPLX, AKC, BKC, 16, G>(p, s);
    }
}

template <bool CPLX, bool AKC, bool BKC, int G> int launch_k(const DmmaParams &p, cudaStream_t s) {
    if constexpr (CPLX) {
        return launch_cfg<CPLX, AKC, BKC, 4, 0>(p, s);  // complex: register budget
    } else {
        return launch_kg<CPLX, AKC, BKC, G>(p, s);
    }
}

template <bool CPLX, int G> int launch_g(const Gemm &g, cudaStream_t s) {
    const DmmaParams p = make_params<CPLX, G>(g);
    if (int64_t(p.tiles_m) * p.tiles_n > INT32_MAX)
        return set_error(BLASX_ERR_UNSUPPORTED, "DMMA grid too large");
    const bool akc = g.ta != NoTrans;  // op(A) = A^T: stored K x M, k contiguous
    const bool bkc = g.tb == NoTrans;  // op(B) = B: stored K x N, k contiguous
    if (akc) return bkc ? launch_k<CPLX, true, true, G>(p, s) : launch_k<CPLX, true, false, G>(p, s);
    return bkc ? launch_k<CPLX, false, true, G>(p, s) : launch_k<CPLX, false, false, G>(p, s);
}

template <bool CPLX> int launch_t(const Gemm &g, cudaStream_t s) {
    if constexpr (CPLX) return launch_g<CPLX, 0>(g, s);
    else return dmma_geometry(g.M, g.N) == 1 ? launch_g<CPLX, 1>(g, s) : launch_g<CPLX, 0>(g, s);
}

}  // namespace

bool dmma_supported(const Gemm &g) {
    return (g.dt == DType::F64 || g.dt == DType::C128) && g.M <= INT32_MAX && g.N <= INT32_MAX &&
           g.K <= INT32_MAX;
}

int launch_gemm_dmma(const Gemm &g, cudaStream_t s) {
    if (g.dt == DType::F64) return launch_t<false>(g, s);
    if (g.dt == DType::C128) return launch_t<true>(g, s);
    return set_error(BLASX_ERR_UNSUPPORTED, "DMMA kernel handles FP64 and complex128 only");
}

}  // namespace bx
