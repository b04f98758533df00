// ozaki.h -- FP64/FP32/complex GEMM emulated with INT8 tensor-core GEMMs
// (Ozaki scheme II: integer scaling + Chinese-remainder reconstruction).
//
// Method (Ozaki, Uchino, Imamura, "Ozaki Scheme II: A GEMM-oriented emulation
// of floating-point matrix multiplication using an integer modular
// technique", 2025), restated for this runtime:
//   1. every row of op(A) and column of op(B) is scaled by a power of two and
//      rounded to an integer (|a'| < 2^62, row 2-norm < 2^Q) so that every
//      dot product of scaled rows is bounded by M/4, M = prod of the moduli;
//   2. for each modulus m_l (pairwise coprime, <= 256) the scaled integers are
//      reduced to symmetric residues in int8;
//   3. one INT8 GEMM per modulus on the tcgen05 tensor cores accumulates in
//      INT32 exactly (|residue| <= 128, K <= 65536); its epilogue reduces the
//      accumulator mod m_l to a uint8 residue;
//   4. the residues are recombined exactly by the CRT in multi-limb integer
//      arithmetic, converted to floating point, unscaled, and the alpha/beta
//      epilogue is applied in FP64.
// The number of moduli is chosen on the device from the measured spread of
// the operands (row/column norm ratios); when no count up to kMaxModuli can
// reach the target accuracy the call falls back to the native FP64 kernel,
// also decided on the device (no host synchronisation).
#pragma once

#include <cstdint>

#include "runtime.h"

namespace bx {
namespace oz {

constexpr int kMaxModuli = 20;
constexpr int kMinModuli = 6;
constexpr int kLimbs = 6;  // 32-bit limbs of CRT weights / products (M < 2^160)
constexpr int kMaxK = 65536;  // INT32-exact accumulation bound (complex uses 2K)

// Padded extents used by the INT8 GEMM tiles.
constexpr int kTileJ = 128;  // MMA M (rows = columns of C)
constexpr int kTileI = 256;  // MMA N (rows of C)
constexpr int kTileK = 128;  // bytes of K per pipeline stage

inline int64_t pad(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Device-side decision record written by the decide kernel.
struct Decision {
    int nmod;      // 0 = native fallback
    int q;         // norm exponent bound Q
    double estimate;  // estimated max normalised error (units of the dtype's u)
    int nonfinite;
    int pad;
};

// Row/column statistics of one operand (R rows of op(X), each over K).
struct RowStats {
    double *amax;    // max |x|
    double *sumsq;   // sum x^2
    double *sumabs;  // sum |x|
    int *flags;      // bit 0: non-finite value seen
};

// INT8 residue GEMM: for every modulus l < *nmod,
//   U_l[j][i] = (sum_k X_l[j][k] * Y_l[i][k]) mod m_l   (uint8, ldu = Ip)
// X: [kMaxModuli][Jp][Kp] int8, Y: [kMaxModuli][Ip][Kp] int8 (K-major).
// Kp multiple of 128, Jp of 128, Ip of 256. Returns a blasx status.
// tj_begin / tj_count: the range of 128-row X tiles (columns of C) to
// compute; tj_count < 0 covers all of them. max_cta_tiles > 0 bounds the
// tiles one CTA computes (more CTAs than SMs, each retiring after a few
// milliseconds); 0 launches one persistent CTA per SM. uplo / diag: only C
// tiles with an entry inside the triangle are computed (row - col <= diag
// for uplo 1, >= diag for 2); jblock: rows of X per column block (Jp for
// real types, half of the stacked complex X).
int launch_residue_gemm(const int8_t *X, const int8_t *Y, uint8_t *U, int64_t Jp, int64_t Ip,
                        int64_t Kp, const Decision *dec, int *err_flag, int num_sms,
                        cudaStream_t s, int64_t tj_begin = 0, int64_t tj_count = -1,
                        int max_cta_tiles = 0, int uplo = 0, int64_t diag = 0, int64_t jblock = 0);

// Host-side CRT constant tables (uploaded once to constant memory).
int upload_crt_tables();

// Uploads the constant tables and sets the kernel attributes of the emulated
// path for the current device (unconditionally; for per-device set-up).
int prepare_crt_tables_current_device();
int prepare_residue_gemm_current_device();

// Test hook of the residue GEMM (blasx_test_stall_residue_gemm): true, with
// the wait limit to use, when the next launch (or executor task) is to stall
// one pipeline stage; each true answer uses up one of the armed stalls.
bool take_residue_stall(long long *wait_cycles);

// The moduli (largest first).
extern const int kModuli[kMaxModuli];

}  // namespace oz

// Whether precision mode `mode` runs g on the emulated path. Mode 2 (ozaki)
// always does when K is within the exact range; mode 1 (native) never; mode
// 0 (auto) where the emulated path measured faster than the native kernels
// on one B200 (device-resident n^3 sweep, 256 <= n <= 4096): FP64 from
// about 1800^3, FP32 from about 640^3, complex128 from about 1200^3. Small K
// also loses: reconstruction costs about as much per C entry as ~350 native
// FP64 multiply-adds, whatever K is.
bool ozaki_selected(const Gemm &g, int mode);

// Emulated GEMM on device-resident operands. Chooses the modulus count on
// the device; falls back to the native kernel on the device when needed.
int ozaki_gemm(const Gemm &g, cudaStream_t s, int mode);

// Scratch bytes the emulated pipeline needs for g, and the pipeline itself
// on a caller-provided scratch of at least that size (allocates nothing;
// the constant tables must already be on the current device).
size_t ozaki_scratch_bytes(const Gemm &g);
int ozaki_gemm_in(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms);

// One K-step of a sequence of emulated GEMMs that share the scratch `ws` in
// stream order (the out-of-core tile steps). The device error flag in the
// scratch is cleared by the first step only, so a bounded-wait failure of
// any step survives to the last one, which copies the flag and the modulus
// decision to the context's host words.
int ozaki_gemm_step(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms, bool first,
                    bool last);

// Column panels of C for the host pipeline: the residue GEMMs and the
// reconstruction run panel by panel (real types; complex runs one panel).
// before_reconstruct(ctx, j0, j1) is called before panel [j0, j1) reads C
// (the host enqueues that panel's copy and makes the stream wait for it);
// after_panel(ctx, j0, j1) once the panel has been enqueued, so that its
// write-back can be ordered behind it. Either may be null.
struct PanelHooks {
    int panels;
    int (*before_reconstruct)(void *ctx, int64_t j0, int64_t j1);
    int (*after_panel)(void *ctx, int64_t j0, int64_t j1);
    void *ctx;
};
// clear_err = false keeps the device error word of earlier calls on the
// same scratch (a sequence of K-blocks accumulating into one C).
int ozaki_gemm_panels(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms,
                      const PanelHooks &hooks, bool clear_err = true);

}  // namespace bx
