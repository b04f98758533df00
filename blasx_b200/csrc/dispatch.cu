// dispatch.cu -- picks the device kernel path for a device-resident GEMM.
//
// Precision mode (blasx_set_dgemm_mode / BLASX_DGEMM_MODE):
//   native  -- FP64 / complex128 on the DMMA kernel, FP32 on the SIMT kernel;
//   auto    -- the INT8 Ozaki path where it measured faster than native
//              (ozaki_selected), K within its exact range; it still falls
//              back to native on the device when the measured spread of the
//              operands needs more than 20 moduli;
//   ozaki   -- the Ozaki path whenever K is within its exact range.
#include <algorithm>

#include "kernels.h"
#include "ozaki.h"
#include "profile.h"

namespace bx {

bool ozaki_selected(const Gemm &g, int mode) {
    const int64_t kmax = is_complex(g.dt) ? oz::kMaxK / 2 : oz::kMaxK;
    if (g.K > kmax || mode == 1) return false;
    if (mode == 2) return true;
    if (std::min(g.M, g.N) < 256) return false;
    const double work = double(g.M) * double(g.N) * double(g.K);
    switch (g.dt) {
        case DType::F64: return g.K >= 512 && work >= 6e9;
        case DType::F32: return g.K >= 256 && work >= 3e8;
        case DType::C64: return g.K >= 256 && work >= 1.5e8;
        default: return g.K >= 256 && work >= 2e9;
    }
}

int device_gemm(const Gemm &g, cudaStream_t s) {
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    if (g.alpha_zero() || g.K == 0) return launch_scale(g, s);
    const int mode = config().dgemm_mode.load();
    if (ozaki_selected(g, mode)) return ozaki_gemm(g, s, mode);
    call_stats().path = 1;
    call_stats().moduli = 0;
    cudaEvent_t e0 = prof::mark(s);
    const int st = dmma_supported(g) ? launch_gemm_dmma(g, s) : launch_gemm_simt(g, s);
    prof::span(prof::kNative, e0, prof::mark(s));
    return st;
}

}  // namespace bx
