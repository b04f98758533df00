// dispatch.cu -- picks the device kernel path for a device-resident GEMM.
#include "kernels.h"

namespace bx {

int device_gemm(const Gemm &g, cudaStream_t s) {
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    if (g.alpha_zero() || g.K == 0) return launch_scale(g, s);
    call_stats().path = 1;
    if (dmma_supported(g)) return launch_gemm_dmma(g, s);
    return launch_gemm_simt(g, s);
}

}  // namespace bx
