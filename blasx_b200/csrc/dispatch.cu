// dispatch.cu -- picks the device kernel path for a device-resident GEMM.
//
// Precision mode (blasx_set_dgemm_mode / BLASX_DGEMM_MODE):
//   native  -- FP64 / complex128 on the DMMA kernel, FP32 on the SIMT kernel;
//   auto    -- the INT8 Ozaki path for problems large enough to amortise its
//              slicing (M*N*K >= 2^27, min(M, N) >= 64), K within its exact
//              range; it still falls back to native on the device when the
//              measured spread of the operands needs more than 20 moduli;
//   ozaki   -- the Ozaki path whenever K is within its exact range.
#include "kernels.h"
#include "ozaki.h"
#include "profile.h"

namespace bx {

namespace {

bool ozaki_k_ok(const Gemm &g) {
    const int64_t kmax = g.dt == DType::C128 ? oz::kMaxK / 2 : oz::kMaxK;
    return g.K <= kmax;
}

bool ozaki_worth_it(const Gemm &g) {
    const double work = double(g.M) * double(g.N) * double(g.K);
    return work >= double(1 << 27) && g.M >= 64 && g.N >= 64 && g.K >= 32;
}

}  // namespace

int device_gemm(const Gemm &g, cudaStream_t s) {
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    if (g.alpha_zero() || g.K == 0) return launch_scale(g, s);
    const int mode = config().dgemm_mode.load();
    const bool oz = ozaki_k_ok(g) && (mode == 2 || (mode == 0 && ozaki_worth_it(g)));
    if (oz) return ozaki_gemm(g, s, mode);
    call_stats().path = 1;
    call_stats().moduli = 0;
    cudaEvent_t e0 = prof::mark(s);
    const int st = dmma_supported(g) ? launch_gemm_dmma(g, s) : launch_gemm_simt(g, s);
    prof::span(prof::kNative, e0, prof::mark(s));
    return st;
}

}  // namespace bx
