// noalloc.cu -- blasx_dgemm_device_noalloc: the emulated DGEMM on
// device-resident operands with its scratch in a fixed device array, so that
// the call allocates no memory at all.
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
// address is looked up with cudaGetSymbolAddress once per device, with that
// device current, on the first call made on that device (which also uploads
// the pipeline's constant tables there), and that address is what the
// kernels receive. All calls share the array and it keeps the last call's
// contents; the pipeline clears what must start at zero (statistics, error
// flag) and overwrites everything else it reads. Calls that overlap on the
// GPU (on different streams, or from several threads) race on the array.
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

// One-time set-up on the current device: device address of the scratch
// array, constant tables and kernel attributes of the emulated pipeline.
int setup_current_device(int dev, void **scratch, int *num_sms) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        BX_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        int sms = 0;
        BX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        BX_TRY(oz::prepare_crt_tables_current_device());
        BX_TRY(oz::prepare_residue_gemm_current_device());
        g_num_sms[dev] = sms;
        g_scratch_addr[dev] = p;
    }
    *scratch = g_scratch_addr[dev];
    *num_sms = g_num_sms[dev];
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
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (g.alpha_zero() || g.K == 0) return launch_scale(g, s);
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
    int dev = 0;
    BX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(BLASX_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    void *scratch = nullptr;
    int num_sms = 0;
    BX_TRY(setup_current_device(dev, &scratch, &num_sms));
    // auto mode: emulated when the operands' spread allows FP64 accuracy,
    // the native FP64 kernel (chosen on the device) otherwise
    return ozaki_gemm_in(g, s, 0, scratch, num_sms);
}
