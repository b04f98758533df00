// runtime.h -- shared types of the B200 GEMM runtime: problem description,
// status recording, the per-process device context and its configuration.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/blasx_b200.h"

namespace bx {

enum class DType : int { F32 = 0, F64 = 1, C128 = 2, C64 = 3 };

inline size_t elem_size(DType t) {
    return t == DType::F32 ? 4 : (t == DType::C128 ? 16 : 8);
}
inline bool is_complex(DType t) { return t == DType::C128 || t == DType::C64; }

struct cplx {
    double re, im;
};

enum Trans : int { NoTrans = 111, TransT = 112, ConjT = 113 };

// How a square operand is stored: the named triangle holds the data, the rest
// is implied (mirrored, conjugate-mirrored, or zero with a stored or unit
// diagonal). SYMM / HEMM operands use the first four, TRMM's diagonal blocks
// the triangular ones.
enum OperandForm : int {
    kGeneral = 0,
    kSymUpper, kSymLower,          // X = X^T
    kHermUpper, kHermLower,        // X = X^H (diagonal imaginary parts are taken as zero)
    kTriUpper, kTriLower,          // zero outside the triangle
    kTriUpperUnit, kTriLowerUnit,  // zero outside, ones on the diagonal
};

// One column-major GEMM C = alpha op(A) op(B) + beta C. Pointers are host or
// device addresses depending on the caller; leading dimensions in elements.
struct Gemm {
    DType dt;
    int ta, tb;
    int64_t M, N, K;
    cplx alpha, beta;
    const void *A;
    int64_t lda;
    const void *B;
    int64_t ldb;
    void *C;
    int64_t ldc;
    // Device pointer; when set, the native kernels return at once unless
    // *guard == 0 (the emulated path chose its native fallback on the device).
    const int *guard = nullptr;
    // Emulated path: at most this many residue-GEMM tiles per CTA (0: one
    // persistent CTA per SM). A bound makes its CTAs retire every few
    // milliseconds, so that kernels of other streams get SMs in between.
    int max_cta_tiles = 0;
    // Triangular output (SYRK): 0 every entry of C; 1 (upper) only entries
    // with row - col <= diag; 2 (lower) only entries with row - col >= diag.
    // Row and column are this GEMM's own C coordinates; diag shifts the
    // diagonal for a block of a larger C. Entries outside are not touched.
    int uplo = 0;
    int64_t diag = 0;
    // Stored form of a square A (or B): only one triangle holds data, and the
    // operand is completed on the device before the product (SYMM, HEMM).
    int a_form = 0, b_form = 0;  // an OperandForm
    // Hermitian output (HERK, HER2K): the imaginary parts of C's diagonal
    // entries (row == col, shifted by diag like uplo) are set to zero once
    // the product is complete.
    bool herm_out = false;

    bool alpha_zero() const { return alpha.re == 0 && alpha.im == 0; }
    bool beta_zero() const { return beta.re == 0 && beta.im == 0; }
    bool beta_one() const { return beta.re == 1 && beta.im == 0; }
    // stored (column-major) shapes of A and B
    int64_t rows_a() const { return ta == NoTrans ? M : K; }
    int64_t cols_a() const { return ta == NoTrans ? K : M; }
    int64_t rows_b() const { return tb == NoTrans ? K : N; }
    int64_t cols_b() const { return tb == NoTrans ? N : K; }
    // whether C entry (r, c) is written
    __host__ __device__ bool in_tri(int64_t r, int64_t c) const {
        return uplo == 0 || (uplo == 1 ? r - c <= diag : r - c >= diag);
    }
    double flops() const {
        return (is_complex(dt) ? 8.0 : 2.0) * double(M) * double(N) * double(K);
    }
};

// One triangular solve with many right-hand sides, column-major: op(A) X =
// alpha B (left) or X op(A) = alpha B (right), X overwriting B (M x N); the
// same fields describe a triangular multiply (TRMM), B = alpha op(A) B or
// alpha B op(A). A is the order-K triangle (K = M left, N right); only its
// `lower` (or upper) triangle is read, and not its diagonal when `unit`.
struct Trsm {
    DType dt;
    bool left, lower, unit;
    int trans;  // NoTrans, TransT, ConjT (ConjT is TransT for real types)
    int64_t M, N;
    cplx alpha;
    const void *A;
    int64_t lda;
    void *B;
    int64_t ldb;
    int64_t order() const { return left ? M : N; }
};

// Records `status` and a formatted message for the calling thread, prints it
// to stderr and returns `status`.
int set_error(int status, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();
int last_status();

#define BX_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t bx_e_ = (call);                                                    \
        if (bx_e_ != cudaSuccess)                                                      \
            return ::bx::set_error(bx_e_ == cudaErrorMemoryAllocation ? BLASX_ERR_NOMEM \
                                                                      : BLASX_ERR_CUDA, \
                                   "%s:%d: %s failed: %s", __FILE__, __LINE__, #call,  \
                                   cudaGetErrorString(bx_e_));                         \
    } while (0)

#define BX_TRY(expr)                     \
    do {                                 \
        int bx_s_ = (expr);              \
        if (bx_s_ != BLASX_OK) return bx_s_; \
    } while (0)

// Library configuration, read once from the environment at first use and
// adjustable through the blasx_set_* calls.
struct Config {
    std::atomic<int> dgemm_mode{0};    // 0 auto, 1 native, 2 ozaki
    std::atomic<size_t> hbm_budget{0}; // 0 = default
    std::atomic<int> tile{0};          // 0 = automatic
    std::atomic<int> host_staging{1};  // pageable host memory: 1 staged, 0 registered
};
Config &config();

// Per-process device state. Created lazily on the first GPU call.
struct Context {
    int device = 0;
    int num_sms = 0;
    size_t total_mem = 0;
    cudaStream_t compute = nullptr;  // kernels
    cudaStream_t h2d = nullptr;      // host -> device copies
    cudaStream_t d2h = nullptr;      // device -> host copies
    std::mutex host_mu;              // serialises host-pipeline calls
    // pinned host slots the emulated path copies its device decision and
    // error flag into (valid once the stream has passed the copy)
    void *last_decision = nullptr;   // oz::Decision
    int *last_error_flag = nullptr;
};

// Returns the context or nullptr (status recorded) when no GPU is usable.
Context *context();
int release_context();

// The reference's info code for a GEMM argument list (0 = legal).
int gemm_arg_info(int order, int ta, int tb, int M, int N, int K, int lda, int ldb, int ldc);

// Counts every kernel launch of the library (blasx_kernel_launch_count).
void count_launch(int n = 1);

// Every device allocation of the library goes through these two. A test hook
// (blasx_test_fail_allocation) can make the n-th one from now report
// cudaErrorMemoryAllocation without allocating, to drive the error paths.
cudaError_t dev_malloc_async(void **p, size_t bytes, cudaStream_t s);
cudaError_t dev_malloc(void **p, size_t bytes);

// Thread-local statistics of the last host call.
blasx_call_stats &call_stats();
// Fills the modulus count / fallback of an emulated call from the pinned
// decision slot (valid once the stream has passed the call).
void resolve_decision(blasx_call_stats &st);

}  // namespace bx
