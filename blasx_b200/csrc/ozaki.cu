// ozaki.cu -- scaling, slicing, modulus-count decision and CRT reconstruction
// of the emulated GEMM (see ozaki.h for the method), and its driver.
//
// Pipeline on one stream, with no host synchronisation:
//   stats(A), stats(B)  -> per-row max|x|, sum x^2, sum |x|, non-finite flag
//   decide              -> modulus count N (0 = native) and norm bound Q
//   slice(A), slice(B)  -> row exponents, int8 residues for l < N
//   residue GEMM        -> uint8 residues of every product (tcgen05)
//   reconstruct         -> exact CRT, unscale, alpha/beta epilogue
//   native guard        -> the native kernel runs only when N == 0
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <type_traits>

#include "kernels.h"
#include "ozaki.h"
#include "ozaki_dev.cuh"
#include "profile.h"

namespace bx {
namespace oz {

const int kModuli[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                 223, 217, 211, 199, 197, 193, 191, 181, 179, 173};

namespace {

// ---- the standalone kernels: one body block per CUDA block -------------------

template <typename T> __global__ void stats_kc_kernel(View v, RowStats st) {
    stats_kc_body<T>(v, st, blockIdx.x, threadIdx.x);
}

template <typename T> __global__ void stats_rc_kernel(View v, RowStats st, int64_t kchunk) {
    stats_rc_body<T>(v, st, kchunk, blockIdx.x, blockIdx.y, threadIdx.x);
}

__global__ void decide_kernel(RowStats sa, int64_t Ra, RowStats sb, int64_t Rb, int64_t K, double unit,
                              int mode, int forced, Decision *dec) {
    decide_body(sa, Ra, sb, Rb, K, unit, mode, forced, dec, threadIdx.x, blockDim.x);
}

template <typename T, int ROLE>
__global__ void __launch_bounds__(256, ROLE == 0 ? 4 : (ROLE == 1 ? 3 : 2)) slice_kc_kernel(View v, RowStats st, const Decision *dec, int *expo,
                                                       SliceOut o) {
    slice_kc_body<T, ROLE>(v, st, dec, expo, o, blockIdx.x, blockIdx.y, threadIdx.x);
}

template <typename T, int ROLE>
__global__ void __launch_bounds__(256, ROLE == 0 ? 4 : (ROLE == 1 ? 3 : 2)) slice_rc_kernel(View v, RowStats st, const Decision *dec, int *expo,
                                                       SliceOut o) {
    __shared__ __align__(16) unsigned char smem[slice_rc_smem_bytes<ROLE>()];
    slice_rc_body<T, ROLE>(v, st, dec, expo, o, blockIdx.x, blockIdx.y, threadIdx.x, smem);
}

template <typename T, bool CPLX>
__global__ void __launch_bounds__(128) reconstruct_kernel(const ReconArgs a, const Decision *dec) {
    reconstruct_body<T, CPLX>(a, dec, blockIdx.x, blockIdx.y, threadIdx.x);
}

std::once_flag g_tables_once;
int g_tables_status = BLASX_OK;

}  // namespace

int upload_crt_tables() {
    std::call_once(g_tables_once, [] {
        if (upload_tables() != cudaSuccess) g_tables_status = BLASX_ERR_CUDA;
    });
    if (g_tables_status != BLASX_OK) return set_error(g_tables_status, "CRT table upload failed");
    return BLASX_OK;
}

int prepare_crt_tables_current_device() {
    BX_CUDA(upload_tables());
    return BLASX_OK;
}

}  // namespace oz

// --------------------------------------------------------------------------
// driver
// --------------------------------------------------------------------------

namespace {

template <typename T>
int launch_stats(const oz::View &v, bool kc, const oz::RowStats &st, cudaStream_t s) {
    if (v.R == 0) return BLASX_OK;
    if (kc) {
        oz::stats_kc_kernel<T><<<unsigned((v.R + 7) / 8), 256, 0, s>>>(v, st);
    } else {
        const int64_t kchunk = 512;
        dim3 grid(unsigned((v.R + 255) / 256), unsigned((v.K + kchunk - 1) / kchunk));
        oz::stats_rc_kernel<T><<<grid, 256, 0, s>>>(v, st, kchunk);
    }
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

template <typename T, int ROLE>
int launch_slice(const oz::View &v, bool kc, const oz::RowStats &st, const oz::Decision *dec,
                 int *expo, const oz::SliceOut &o, int64_t Kc, cudaStream_t s) {
    if (kc) {
        dim3 grid(unsigned(Kc / 64), unsigned(o.Rp / 64));
        oz::slice_kc_kernel<T, ROLE><<<grid, 256, 0, s>>>(v, st, dec, expo, o);
    } else {
        const int kt = ROLE ? 32 : 64;
        dim3 grid(unsigned(Kc / kt), unsigned(o.Rp / 64));
        oz::slice_rc_kernel<T, ROLE><<<grid, 256, 0, s>>>(v, st, dec, expo, o);
    }
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

// The whole emulated pipeline on a caller-provided workspace of
// make_plan(g).bytes bytes: no allocation. The device decision and error
// flag are copied to the given host slots when they are not null.
template <typename T>
int ozaki_run(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms, void *dec_host,
              int *err_host, const PanelHooks *hooks = nullptr, bool clear_err = true) {
    constexpr bool CPLX = oz::Elem<T>::cplx;
    const oz::Plan pl = oz::make_plan(g);
    const int64_t M = pl.M, N = pl.N, K = pl.K, Kh = pl.Kh, Kp = pl.Kp, Kc = pl.Kc;
    const int64_t Ip = pl.Ip, Jp = pl.Jp, Jx = pl.Jx;
    const oz::Parts pt = oz::carve_parts(g, pl, ws);
    int *err = pt.err;
    oz::Decision *dec = pt.dec;
    const oz::RowStats sa = pt.sa, sb = pt.sb;
    int *ea = pt.ea, *fb = pt.fb;
    int8_t *Y = pt.Y, *X = pt.X;
    uint8_t *U = pt.U;
    const size_t stats_bytes = pt.stats_bytes;
    cudaEvent_t ev0 = prof::mark(s);
    BX_CUDA(cudaMemsetAsync(sa.amax, 0, stats_bytes, s));
    if (clear_err) BX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));

    // op(A) rows i over k; op(B) columns j over k
    oz::View va{g.A, g.lda, M, K, g.ta == ConjT};
    oz::View vb{g.B, g.ldb, N, K, g.tb == ConjT};
    const bool akc = g.ta != NoTrans, bkc = g.tb == NoTrans;
    BX_TRY(launch_stats<T>(va, akc, sa, s));
    if (!pl.alias) BX_TRY(launch_stats<T>(vb, bkc, sb, s));
    const oz::RowStats sbd = pl.alias ? sa : sb;  // aliased: the columns of op(B) are the rows of op(A)
    int *fbd = pl.alias ? ea : fb;
    const double unit = oz::Elem<T>::single ? std::ldexp(1.0, -24) : std::ldexp(1.0, -53);
    oz::decide_kernel<<<1, 1024, 0, s>>>(sa, M, sbd, N, K, unit, mode, oz::forced_moduli(), dec);
    BX_CUDA(cudaGetLastError());
    count_launch();

    oz::SliceOut oy{Y, Ip, Kp, Kh, Ip * Kp};
    oz::SliceOut ox{X, Jp, Kp, Kh, Jx * Kp};
    if constexpr (CPLX) {
        BX_TRY((launch_slice<T, 1>(va, akc, sa, dec, ea, oy, Kc, s)));
        BX_TRY((launch_slice<T, 2>(vb, bkc, sb, dec, fb, ox, Kc, s)));
    } else {
        BX_TRY((launch_slice<T, 0>(va, akc, sa, dec, ea, oy, Kc, s)));
        if (!pl.alias) BX_TRY((launch_slice<T, 0>(vb, bkc, sb, dec, fb, ox, Kc, s)));
    }
    // residue GEMMs and reconstruction, in column panels of C when asked.
    // (Running a panel's reconstruction on a second stream beside the next
    // panel's residue GEMM was measured slower: under the power cap the
    // concurrent integer work lowers the clock of the tensor work.)
    const int64_t tiles_j = Jp / oz::kTileJ;
    const int panels = (CPLX || !hooks) ? 1 : int(std::max<int64_t>(1, std::min<int64_t>(hooks->panels, tiles_j)));
    cudaEvent_t ev1 = prof::mark(s), ev2 = nullptr;
    for (int pnl = 0; pnl < panels; ++pnl) {
        const int64_t tj0 = tiles_j * pnl / panels, tj1 = tiles_j * (pnl + 1) / panels;
        const int64_t j0 = tj0 * oz::kTileJ, j1 = std::min<int64_t>(N, tj1 * oz::kTileJ);
        if (panels == 1) {
            BX_TRY(oz::launch_residue_gemm(X, Y, U, Jx, Ip, Kp, dec, err, num_sms, s, 0, -1, g.max_cta_tiles,
                                           g.uplo, g.diag, Jp));
        } else {
            BX_TRY(oz::launch_residue_gemm(X, Y, U, Jx, Ip, Kp, dec, err, num_sms, s, tj0, tj1 - tj0,
                                           g.max_cta_tiles, g.uplo, g.diag, Jp));
        }
        if (pnl == 0) ev2 = prof::mark(s);
        if (hooks && hooks->before_reconstruct && j1 > j0)
            BX_TRY(hooks->before_reconstruct(hooks->ctx, j0, j1));
        // grid.y is limited to 65535 columns per launch
        for (int64_t c0 = j0; c0 < j1; c0 += 65535) {
            const int64_t c1 = std::min<int64_t>(j1, c0 + 65535);
            dim3 rgrid(unsigned((M + 4 * 128 - 1) / (4 * 128)), unsigned(c1 - c0));
            oz::ReconArgs ra{U, Jp, Ip, M, N, ea, fbd, g.alpha.re, g.alpha.im, g.beta.re, g.beta.im,
                             g.beta_zero() ? 1 : 0, g.C, g.ldc, c0, g.uplo, g.diag};
            oz::reconstruct_kernel<T, CPLX><<<rgrid, 128, 0, s>>>(ra, dec);
            BX_CUDA(cudaGetLastError());
            count_launch();
        }
        if (hooks && j1 > j0) {
            // native fallback for this panel's columns (runs only when nmod == 0),
            // so that the panel's write-back also follows the fallback
            Gemm gp = g;
            gp.N = j1 - j0;
            gp.B = static_cast<const char *>(g.B) +
                   (g.tb == NoTrans ? j0 * g.ldb : j0) * int64_t(elem_size(g.dt));
            gp.C = static_cast<char *>(g.C) + j0 * g.ldc * int64_t(elem_size(g.dt));
            gp.diag = g.diag + j0;
            gp.guard = &dec->nmod;
            if (dmma_supported(gp)) BX_TRY(launch_gemm_dmma(gp, s));
            else BX_TRY(launch_gemm_simt(gp, s));
        }
        if (hooks && hooks->after_panel) BX_TRY(hooks->after_panel(hooks->ctx, j0, j1));
    }
    cudaEvent_t ev3 = prof::mark(s);

    // native fallback, decided on the device (runs only when nmod == 0);
    // with panels it already ran panel by panel
    if (!hooks) {
        Gemm gn = g;
        gn.guard = &dec->nmod;
        if (dmma_supported(gn)) BX_TRY(launch_gemm_dmma(gn, s));
        else BX_TRY(launch_gemm_simt(gn, s));
    }
    cudaEvent_t ev4 = prof::mark(s);
    prof::span(prof::kSlice, ev0, ev1);
    prof::span(prof::kResidueGemm, ev1, ev2);
    prof::span(prof::kReconstruct, ev2, ev3);
    prof::span(prof::kNative, ev3, ev4);

    // record the decision for blasx_get_call_stats (lands when the stream does)
    if (dec_host)
        BX_CUDA(cudaMemcpyAsync(dec_host, dec, sizeof(oz::Decision), cudaMemcpyDeviceToHost, s));
    if (err_host) BX_CUDA(cudaMemcpyAsync(err_host, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    call_stats().path = 2;
    call_stats().moduli = -1;  // decided on the device: resolved from dec_host once the stream has passed
    return BLASX_OK;
}

template <typename T> int ozaki_t(const Gemm &g, cudaStream_t s, int mode) {
    Context *ctx = context();
    if (!ctx) return last_status();
    BX_TRY(oz::upload_crt_tables());
    const oz::Plan pl = oz::make_plan(g);
    void *ws = nullptr;
    BX_CUDA(dev_malloc_async(&ws, pl.bytes, s));
    struct Free {
        void *p;
        cudaStream_t s;
        ~Free() { cudaFreeAsync(p, s); }
    } free_ws{ws, s};
    return ozaki_run<T>(g, s, mode, ws, ctx->num_sms, ctx->last_decision, ctx->last_error_flag);
}

}  // namespace

int ozaki_gemm(const Gemm &g, cudaStream_t s, int mode) {
    switch (g.dt) {
        case DType::F64: return ozaki_t<double>(g, s, mode);
        case DType::F32: return ozaki_t<float>(g, s, mode);
        case DType::C64: return ozaki_t<oz::cpair>(g, s, mode);
        default: return ozaki_t<oz::zpair>(g, s, mode);
    }
}

size_t ozaki_scratch_bytes(const Gemm &g) { return oz::make_plan(g).bytes; }

int ozaki_gemm_panels(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms,
                      const PanelHooks &hooks, bool clear_err) {
    Context *ctx = context();
    if (!ctx) return last_status();
    BX_TRY(oz::upload_crt_tables());
    switch (g.dt) {
        case DType::F64:
            return ozaki_run<double>(g, s, mode, ws, num_sms, ctx->last_decision, ctx->last_error_flag, &hooks,
                                     clear_err);
        case DType::C64:
            return ozaki_run<oz::cpair>(g, s, mode, ws, num_sms, ctx->last_decision, ctx->last_error_flag, &hooks,
                                        clear_err);
        case DType::F32:
            return ozaki_run<float>(g, s, mode, ws, num_sms, ctx->last_decision, ctx->last_error_flag, &hooks,
                                    clear_err);
        default:
            return ozaki_run<oz::zpair>(g, s, mode, ws, num_sms, ctx->last_decision, ctx->last_error_flag,
                                        &hooks, clear_err);
    }
}

int ozaki_gemm_step(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms, bool first,
                    bool last) {
    Context *ctx = context();
    if (!ctx) return last_status();
    BX_TRY(oz::upload_crt_tables());
    void *dec_host = last ? ctx->last_decision : nullptr;
    int *err_host = last ? ctx->last_error_flag : nullptr;
    switch (g.dt) {
        case DType::F64: return ozaki_run<double>(g, s, mode, ws, num_sms, dec_host, err_host, nullptr, first);
        case DType::F32: return ozaki_run<float>(g, s, mode, ws, num_sms, dec_host, err_host, nullptr, first);
        case DType::C64: return ozaki_run<oz::cpair>(g, s, mode, ws, num_sms, dec_host, err_host, nullptr, first);
        default: return ozaki_run<oz::zpair>(g, s, mode, ws, num_sms, dec_host, err_host, nullptr, first);
    }
}

int ozaki_gemm_in(const Gemm &g, cudaStream_t s, int mode, void *ws, int num_sms) {
    switch (g.dt) {
        case DType::F64: return ozaki_run<double>(g, s, mode, ws, num_sms, nullptr, nullptr);
        case DType::F32: return ozaki_run<float>(g, s, mode, ws, num_sms, nullptr, nullptr);
        case DType::C64: return ozaki_run<oz::cpair>(g, s, mode, ws, num_sms, nullptr, nullptr);
        default: return ozaki_run<oz::zpair>(g, s, mode, ws, num_sms, nullptr, nullptr);
    }
}

}  // namespace bx
