// noalloc.cu -- blasx_dgemm_device_noalloc: the emulated DGEMM on
// device-resident operands with its scratch in a fixed device array, so that
// the call allocates no memory at all; and blasx_dgemm_device_noalloc_status,
// which reads that scratch's device error word back.
//
// Some callers cannot let a library call cudaMalloc: a framework whose
// caching allocator has already reserved the GPU's memory (a cudaMalloc
// there fails or fragments its pool), and latency-critical code where
// cudaMalloc / cudaFree may synchronise the device. This entry point serves
// them: the caller passes inputs and outputs, and every byte of scratch the
// emulated pipeline needs (row statistics, the modulus decision, int8
// slices, uint8 residues) is carved out of kScratchBytes of statically
// allocated device memory, which every GPU that loads the library holds
// until the process exits.
//
// The array's name is only a host-side stand-in in host code: its device
// address is looked up with cudaGetSymbolAddress once per device context,
// with that device current, on the first call made there (which also
// uploads the pipeline's constant tables and kernel attributes), and that
// address is what the kernels receive. The set-up is redone when the
// device's current context is a different one (after cudaDeviceReset). All
// calls share the array and it keeps the last call's contents; the pipeline
// clears what must start at zero (statistics, error word) and overwrites
// everything else it reads. Calls that overlap on the GPU (on different
// streams, or from several threads) race on the array.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "kernels.h"
#include "ozaki.h"

namespace bx {
namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
void *g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};
unsigned long long g_ctx_id[kMaxDevices] = {};

// Unique id of the calling thread's current context (0 when there is none or
// the driver cannot tell). Context handles can be reused after a reset; the
// ids of cuCtxGetId are not.
unsigned long long current_context_id() {
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Set-up on the current device, once per context: device address of the
// scratch array, constant tables and kernel attributes of the emulated
// pipeline. When the driver cannot report a context id, the set-up runs once
// per device.
int setup_current_device(int dev, void **scratch, int *num_sms) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    const unsigned long long id = current_context_id();
    if (!g_scratch_addr[dev] || (id != 0 && id != g_ctx_id[dev])) {
        void *p = nullptr;
        BX_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        int sms = 0;
        BX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        BX_TRY(oz::prepare_crt_tables_current_device());
        BX_TRY(oz::prepare_residue_gemm_current_device());
        g_num_sms[dev] = sms;
        g_scratch_addr[dev] = p;
        // the symbol lookup made the runtime's context current if none was
        g_ctx_id[dev] = id ? id : current_context_id();
    }
    *scratch = g_scratch_addr[dev];
    *num_sms = g_num_sms[dev];
    return BLASX_OK;
}

int current_device(int *dev) {
    BX_CUDA(cudaGetDevice(dev));
    if (*dev < 0 || *dev >= kMaxDevices)
        return set_error(BLASX_ERR_UNSUPPORTED, "device ordinal %d out of range", *dev);
    return BLASX_OK;
}

}  // namespace
}  // namespace bx

extern "C" int blasx_dgemm_device_noalloc(int transa, int transb, int M, int N, int K,
                                          double alpha, const double *A, int lda,
                                          const double *B, int ldb, double beta, double *C,
                                          int ldc, void *stream) {
    using namespace bx;
    clear_error();
    const int info = gemm_arg_info(CblasColMajor, transa, transb, M, N, K, lda, ldb, ldc);
    if (info) return set_error(BLASX_ERR_ARG, "no-alloc dgemm parameter %d illegal", info);
    Gemm g;
    g.dt = DType::F64;
    g.ta = transa == ConjT ? TransT : transa;
    g.tb = transb == ConjT ? TransT : transb;
    g.M = M; g.N = N; g.K = K;
    g.alpha = cplx{alpha, 0}; g.beta = cplx{beta, 0};
    g.A = A; g.lda = lda; g.B = B; g.ldb = ldb; g.C = C; g.ldc = ldc;
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    const int mode = config().dgemm_mode.load();
    const bool emulate = mode != 1 && !g.alpha_zero() && g.K != 0;
    if (emulate) {
        if (g.K > oz::kMaxK)
            return set_error(BLASX_ERR_UNSUPPORTED,
                             "blasx_dgemm_device_noalloc: K=%d exceeds the emulated path's limit %d",
                             K, oz::kMaxK);
        const size_t need = ozaki_scratch_bytes(g);
        if (need > kScratchBytes)
            return set_error(BLASX_ERR_UNSUPPORTED,
                             "blasx_dgemm_device_noalloc: M=%d N=%d K=%d needs %zu bytes of scratch; "
                             "the static scratch holds %zu bytes (M=N=K=1024 fits)",
                             M, N, K, need, kScratchBytes);
    }
    int dev = 0;
    BX_TRY(current_device(&dev));
    void *scratch = nullptr;
    int num_sms = 0;
    BX_TRY(setup_current_device(dev, &scratch, &num_sms));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!emulate) {
        // no scratch is used: clear the error word so that the status query
        // does not report an earlier call's failure for this one
        BX_CUDA(cudaMemsetAsync(scratch, 0, sizeof(int), s));
        if (g.alpha_zero() || g.K == 0) return launch_scale(g, s);
        return launch_gemm_dmma(g, s);
    }
    // auto mode: emulated when the operands' spread allows FP64 accuracy, the
    // native FP64 kernel (chosen on the device) otherwise; ozaki mode: always
    // emulated. The pipeline clears the scratch's error word (its first
    // word) and raises it when a bounded device wait ran out.
    return ozaki_gemm_in(g, s, mode, scratch, num_sms);
}

extern "C" int blasx_dgemm_device_noalloc_status(void *stream) {
    using namespace bx;
    clear_error();
    int dev = 0;
    BX_TRY(current_device(&dev));
    void *scratch = nullptr;
    int num_sms = 0;
    BX_TRY(setup_current_device(dev, &scratch, &num_sms));
    BX_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    int word = 0;
    BX_CUDA(cudaMemcpy(&word, scratch, sizeof(int), cudaMemcpyDeviceToHost));
    if (word)
        return set_error(BLASX_ERR_TIMEOUT,
                         "blasx_dgemm_device_noalloc: a bounded wait of the residue GEMM ran out "
                         "(error word 0x%x); C is undefined", word);
    return BLASX_OK;
}
