// kernels_sgemm.cu -- FP32 GEMM on the CUDA cores for problems that fill the
// GPU: the 128 x 128 tile of simt_tile.cuh, one CTA per C tile.
#include "kernels.h"
#include "simt_tile.cuh"

namespace bx {
namespace {

using namespace dev;

__global__ void __launch_bounds__(sg::THR, 2) sgemm128_kernel(const SimtParams<float> p, const int *guard) {
    if (guard && *guard != 0) return;  // the emulated path produced C
    __shared__ __align__(16) float smem[sgemm128_smem_bytes() / sizeof(float)];
    sgemm128_tile(p, blockIdx.x, blockIdx.y, smem);
}

}  // namespace

bool sgemm128_fits(const Gemm &g) {
    using namespace dev::sg;
    const int64_t tiles = ((g.M + TM - 1) / TM) * ((g.N + TN - 1) / TN);
    return g.dt == DType::F32 && tiles >= 148 && g.M <= INT32_MAX && g.N <= INT32_MAX && g.K <= INT32_MAX &&
           (g.N + TN - 1) / TN <= 65535;
}

int launch_sgemm128(const Gemm &g, cudaStream_t s) {
    using namespace dev::sg;
    dim3 grid(unsigned((g.M + TM - 1) / TM), unsigned((g.N + TN - 1) / TN));
    const SimtParams<float> p{g.ta, g.tb, int(g.M), int(g.N), int(g.K), float(g.alpha.re), float(g.beta.re),
                              static_cast<const float *>(g.A), g.lda, static_cast<const float *>(g.B), g.ldb,
                              static_cast<float *>(g.C), g.ldc, g.beta_zero() ? 1 : 0, g.uplo, g.diag};
    sgemm128_kernel<<<grid, sg::THR, 0, s>>>(p, g.guard);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

}  // namespace bx
