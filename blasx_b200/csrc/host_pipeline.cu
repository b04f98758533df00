// host_pipeline.cu -- GEMM on host-resident operands.
//
// Replaces the reference's per-call flow (blas/dgemm.c:88-121: pin A/B/C,
// build per-GPU caches, run the tiled runtime, unpin) with two paths:
//
//   in-core   A, B, C (and the emulated path's scratch) fit the HBM budget:
//             C is processed in column panels. The H2D stream copies A, then
//             for every panel its B columns (and C columns when beta != 0);
//             the compute stream runs the panel as soon as its operands have
//             landed; the D2H stream writes the panel back while later panels
//             compute. The emulated path slices A and B once (its statistics
//             need the whole operands), then runs the residue GEMMs and the
//             reconstruction panel by panel with the same write-back overlap.
//             With K >= 4096 it works in two K-blocks: block 1 is sliced and
//             multiplied while block 2's A and B are still on the host link,
//             C0 comes last and is added panel by panel (beta C0).
//   tiled     otherwise: the HBM tile cache with an explicit byte budget
//             (tile_engine.cu), native kernels.
//
// Host buffers that are not pinned are staged through pinned bounce buffers
// (staging.h), or registered for the call (full ld x columns extent) when
// staging is switched off, so that every copy is an asynchronous DMA.
#include <algorithm>
#include <chrono>
#include <vector>

#include "host_pipeline.h"
#include "kernels.h"
#include "ozaki.h"
#include "tile_engine.h"

namespace bx {

namespace {

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

struct Events {
    std::vector<cudaEvent_t> evs;
    ~Events() {
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
    }
    cudaEvent_t make() {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) evs.push_back(e);
        return e;
    }
};

// Device copies of the operands, laid out column-major with ld padded to 32.
struct DeviceOps {
    void *A = nullptr, *B = nullptr, *C = nullptr, *ws = nullptr;
    void *C0 = nullptr;  // input C, when the emulated path accumulates K-blocks into C
    void *diag = nullptr;  // TRMM: one completed diagonal block
    bool b_is_a = false;  // B is the same host buffer as A (SYRK): one device copy
    int64_t lda = 0, ldb = 0, ldc = 0;
    cudaStream_t s = nullptr;
    ~DeviceOps() {
        for (void *p : {A, b_is_a ? nullptr : B, C, ws, C0, diag})
            if (p) cudaFreeAsync(p, s);
    }
};

// B read from A's host buffer with the same stored shape (SYRK's op(A) op(A)^T).
bool b_is_a(const Gemm &g) {
    return g.A == g.B && g.lda == g.ldb && g.rows_a() == g.rows_b() && g.cols_a() == g.cols_b();
}

size_t default_budget(const Context *c) {
    size_t b = config().hbm_budget.load();
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return b ? b : c->total_mem / 2;
    // the tile arena the library already holds is reusable, count it as free
    const size_t cap = size_t(double(free_b) * 0.9);
    return b ? std::min(b, total_b) : cap;
}

size_t tile_step_ws(const Gemm &g, int T, int mode);

// Tile edge of the out-of-core path: BLASX_TILE / blasx_set_tile when set;
// otherwise 4096 (complex128: 2048), or twice that when the K-steps of that
// edge run emulated and the budget holds 16 operand tiles of it beside the C
// tiles and the step scratch. An emulated K-step slices its tiles and
// reconstructs its C tile every time, work that a larger edge spreads over
// more multiply-adds (40960^3 through a 24 GiB cache: 1.18 s at 8192 against
// 1.51 s at 4096); native K-steps peak at 4096.
int pick_tile(const Gemm &g, int mode, size_t budget) {
    const int t = config().tile.load();
    if (t) return t;
    const int base = g.dt == DType::C128 ? 2048 : 4096, big = 2 * base;
    const size_t ws = tile_step_ws(g, big, mode);
    const size_t slot = size_t(big) * big * elem_size(g.dt);
    if (ws && budget >= tiled_min_bytes(g.dt, big, ws) + 14 * slot) return big;
    return base;
}

// Copies the column panel [j0, j1) of op(B) (and of C) host -> device.
int copy_panel_in(const Gemm &g, const DeviceOps &d, int64_t j0, int64_t j1, bool need_b,
                  bool read_c, cudaStream_t s, blasx_call_stats &st) {
    const size_t es = elem_size(g.dt);
    const int64_t w = j1 - j0;
    if (need_b && !d.b_is_a) {
        const char *hb = static_cast<const char *>(g.B);
        char *db = static_cast<char *>(d.B);
        if (g.tb == NoTrans) {  // K x N stored: columns j0..j1
            BX_TRY(copy2d(db + j0 * d.ldb * es, d.ldb * es, hb + j0 * g.ldb * es,
                                      g.ldb * es, g.K * es, w, cudaMemcpyHostToDevice, s));
        } else {  // N x K stored: rows j0..j1
            BX_TRY(copy2d(db + j0 * es, d.ldb * es, hb + j0 * es, g.ldb * es, w * es,
                                      g.K, cudaMemcpyHostToDevice, s));
        }
        st.h2d_bytes += double(w) * g.K * es;
    }
    if (read_c) {
        BX_TRY(copy2d(static_cast<char *>(d.C) + j0 * d.ldc * es, d.ldc * es,
                                  static_cast<const char *>(g.C) + j0 * g.ldc * es, g.ldc * es,
                                  g.M * es, w, cudaMemcpyHostToDevice, s));
        st.h2d_bytes += double(w) * g.M * es;
    }
    return BLASX_OK;
}

int copy_panel_out(const Gemm &g, const DeviceOps &d, int64_t j0, int64_t j1, cudaStream_t s,
                   blasx_call_stats &st) {
    const size_t es = elem_size(g.dt);
    BX_TRY(copy2d(static_cast<char *>(g.C) + j0 * g.ldc * es, g.ldc * es,
                              static_cast<const char *>(d.C) + j0 * d.ldc * es, d.ldc * es,
                              g.M * es, j1 - j0, cudaMemcpyDeviceToHost, s));
    st.d2h_bytes += double(j1 - j0) * g.M * es;
    return BLASX_OK;
}

int panel_count(const Gemm &g) {
    // panels of >= 1024 columns, at most 16: the last panel's copies are
    // the pipeline's exposed tail
    return int(std::max<int64_t>(1, std::min<int64_t>(16, g.N / 1024)));
}

// ---- operands stored as one triangle (SYMM, HEMM) ---------------------------
// Gemm::a_form / b_form name the stored triangle of a square operand. Its
// device copy lands whole; complete_forms then fills in the rest in place
// (mirror or conjugate mirror) before any GEMM reads it.

int complete_forms(const Gemm &g, const DeviceOps &d, cudaStream_t s) {
    BX_TRY(launch_complete_operand(g.dt, g.a_form, d.A, d.lda, g.rows_a(), s));
    return launch_complete_operand(g.dt, g.b_form, d.B, d.ldb, g.rows_b(), s);
}

// ---- in-core, native kernels ----------------------------------------------
int incore_native(const Gemm &g, Context *c, DeviceOps &d, bool need_ab, bool read_c,
                  blasx_call_stats &st) {
    Events ev;
    const size_t es = elem_size(g.dt);
    cudaEvent_t start = ev.make();
    BX_CUDA(cudaEventRecord(start, c->compute));  // device buffers allocated on compute
    BX_CUDA(cudaStreamWaitEvent(c->h2d, start, 0));
    BX_CUDA(cudaStreamWaitEvent(c->d2h, start, 0));
    if (need_ab) {
        BX_TRY(copy2d(d.A, d.lda * es, g.A, g.lda * es, g.rows_a() * es, g.cols_a(),
                                  cudaMemcpyHostToDevice, c->h2d));
        st.h2d_bytes += double(es) * g.rows_a() * g.cols_a();
        if (g.b_form) {  // a stored triangle is completed whole: B lands before the panels
            BX_TRY(copy2d(d.B, d.ldb * es, g.B, g.ldb * es, g.rows_b() * es, g.cols_b(),
                                      cudaMemcpyHostToDevice, c->h2d));
            st.h2d_bytes += double(es) * g.rows_b() * g.cols_b();
        }
    }
    const int panels = panel_count(g);
    for (int p = 0; p < panels; ++p) {
        const int64_t j0 = g.N * p / panels, j1 = g.N * (p + 1) / panels;
        BX_TRY(copy_panel_in(g, d, j0, j1, need_ab && !g.b_form, read_c, c->h2d, st));
        cudaEvent_t in = ev.make();
        BX_CUDA(cudaEventRecord(in, c->h2d));
        BX_CUDA(cudaStreamWaitEvent(c->compute, in, 0));
        if (p == 0 && need_ab) BX_TRY(complete_forms(g, d, c->compute));
        Gemm p_g = g;
        p_g.N = j1 - j0;
        p_g.A = d.A; p_g.lda = d.lda;
        p_g.B = static_cast<char *>(d.B) + (g.tb == NoTrans ? j0 * d.ldb : j0) * es;
        p_g.ldb = d.ldb;
        p_g.C = static_cast<char *>(d.C) + j0 * d.ldc * es;
        p_g.ldc = d.ldc;
        p_g.diag = g.diag + j0;  // triangular output: this panel's columns start at j0
        if (need_ab) {
            BX_TRY(dmma_supported(p_g) ? launch_gemm_dmma(p_g, c->compute)
                                       : launch_gemm_simt(p_g, c->compute));
        } else {
            BX_TRY(launch_scale(p_g, c->compute));
        }
        if (g.herm_out) BX_TRY(launch_real_diagonal(g.dt, p_g.C, d.ldc, g.M, j1 - j0, j0 + g.diag, c->compute));
        cudaEvent_t done = ev.make();
        BX_CUDA(cudaEventRecord(done, c->compute));
        BX_CUDA(cudaStreamWaitEvent(c->d2h, done, 0));
        BX_TRY(copy_panel_out(g, d, j0, j1, c->d2h, st));
    }
    BX_CUDA(cudaStreamSynchronize(c->h2d));
    BX_CUDA(cudaStreamSynchronize(c->compute));
    BX_CUDA(cudaStreamSynchronize(c->d2h));
    st.path = need_ab ? 1 : 3;
    return BLASX_OK;
}

// ---- in-core, emulated path -------------------------------------------------
struct OzPanelCtx {
    const Gemm *g;
    const DeviceOps *d;
    Context *c;
    Events *ev;
    blasx_call_stats *st;
};

int oz_after_panel(void *vctx, int64_t j0, int64_t j1) {
    auto *x = static_cast<OzPanelCtx *>(vctx);
    if (x->g->herm_out)
        BX_TRY(launch_real_diagonal(x->g->dt, static_cast<char *>(x->d->C) + j0 * x->d->ldc * elem_size(x->g->dt),
                                    x->d->ldc, x->g->M, j1 - j0, j0 + x->g->diag, x->c->compute));
    cudaEvent_t done = x->ev->make();
    BX_CUDA(cudaEventRecord(done, x->c->compute));
    BX_CUDA(cudaStreamWaitEvent(x->c->d2h, done, 0));
    return copy_panel_out(*x->g, *x->d, j0, j1, x->c->d2h, *x->st);
}

// C panel copy-in, queued behind A and B on the H2D stream; only this
// panel's reconstruction waits for it.
int oz_before_reconstruct(void *vctx, int64_t j0, int64_t j1) {
    auto *x = static_cast<OzPanelCtx *>(vctx);
    BX_TRY(copy_panel_in(*x->g, *x->d, j0, j1, false, true, x->c->h2d, *x->st));
    cudaEvent_t in = x->ev->make();
    BX_CUDA(cudaEventRecord(in, x->c->h2d));
    BX_CUDA(cudaStreamWaitEvent(x->c->compute, in, 0));
    return BLASX_OK;
}

// K-blocks of the emulated in-core path: op(A)(:, k0:k1) and op(B)(k0:k1, :)
// are copied block by block, so that block b computes while block b + 1 is
// on the host link. Two blocks once K >= 4096 (each block's slicing and
// residue GEMMs are independent; the blocks' results are summed in FP64).
int kblock_count(const Gemm &g) {
    // a triangular output keeps one block: its panels read C whole before
    // reconstructing into it, so the other triangle goes back unchanged
    return g.K >= 4096 && g.uplo == 0 ? 2 : 1;
}

int64_t kblock_edge(const Gemm &g, int b, int blocks) {
    return b == blocks ? g.K : (g.K * b / blocks) / 128 * 128;
}

// The block's view of a GEMM whose A and B start at a, b with leading
// dimensions lda, ldb (host or device copies alike).
Gemm kblock_of(const Gemm &g, const void *a, int64_t lda, const void *b, int64_t ldb, int64_t k0,
               int64_t k1) {
    const size_t es = elem_size(g.dt);
    Gemm k = g;
    k.K = k1 - k0;
    k.A = static_cast<const char *>(a) + (g.ta == NoTrans ? k0 * lda : k0) * int64_t(es);
    k.lda = lda;
    k.B = static_cast<const char *>(b) + (g.tb == NoTrans ? k0 : k0 * ldb) * int64_t(es);
    k.ldb = ldb;
    return k;
}

int copy_kblock_in(const Gemm &g, const DeviceOps &d, int64_t k0, int64_t k1, cudaStream_t s,
                   blasx_call_stats &st) {
    const size_t es = elem_size(g.dt);
    const Gemm h = kblock_of(g, g.A, g.lda, g.B, g.ldb, k0, k1);
    const Gemm v = kblock_of(g, d.A, d.lda, d.B, d.ldb, k0, k1);
    BX_TRY(copy2d(const_cast<void *>(v.A), d.lda * es, h.A, g.lda * es, h.rows_a() * es,
                              h.cols_a(), cudaMemcpyHostToDevice, s));
    if (!d.b_is_a)
        BX_TRY(copy2d(const_cast<void *>(v.B), d.ldb * es, h.B, g.ldb * es, h.rows_b() * es,
                                  h.cols_b(), cudaMemcpyHostToDevice, s));
    st.h2d_bytes += double(es) * (h.rows_a() * h.cols_a() + (d.b_is_a ? 0 : h.rows_b() * h.cols_b()));
    return BLASX_OK;
}

// Last K-block, per C panel: C0 panel in (beta != 0), C += beta C0, write-back.
int oz_after_panel_kblocks(void *vctx, int64_t j0, int64_t j1) {
    auto *x = static_cast<OzPanelCtx *>(vctx);
    const Gemm &g = *x->g;
    const DeviceOps &d = *x->d;
    const size_t es = elem_size(g.dt);
    if (!g.beta_zero()) {
        BX_TRY(copy2d(static_cast<char *>(d.C0) + j0 * d.ldc * es, d.ldc * es,
                                  static_cast<const char *>(g.C) + j0 * g.ldc * es, g.ldc * es,
                                  g.M * es, j1 - j0, cudaMemcpyHostToDevice, x->c->h2d));
        x->st->h2d_bytes += double(j1 - j0) * g.M * es;
        cudaEvent_t in = x->ev->make();
        BX_CUDA(cudaEventRecord(in, x->c->h2d));
        BX_CUDA(cudaStreamWaitEvent(x->c->compute, in, 0));
        Gemm p = g;
        p.N = j1 - j0;
        p.C = static_cast<char *>(d.C) + j0 * d.ldc * es;
        p.ldc = d.ldc;
        p.diag = g.diag + j0;
        BX_TRY(launch_add_scaled(p, static_cast<const char *>(d.C0) + j0 * d.ldc * es, d.ldc,
                                 x->c->compute));
    }
    return oz_after_panel(vctx, j0, j1);
}

int finish_ozaki(Context *c, blasx_call_stats &st) {
    BX_CUDA(cudaStreamSynchronize(c->h2d));
    BX_CUDA(cudaStreamSynchronize(c->compute));
    BX_CUDA(cudaStreamSynchronize(c->d2h));
    st.path = 2;
    resolve_decision(st);
    if (*c->last_error_flag)
        return set_error(BLASX_ERR_TIMEOUT, "emulated GEMM: bounded device wait expired (flag %d)",
                         *c->last_error_flag);
    return BLASX_OK;
}

// Emulated path in K-blocks: every block's A and B columns / rows go first on
// the H2D stream, C0 (beta != 0) after all of them. Block b computes
// C = alpha op(A_b) op(B_b) + (b ? C : 0) as soon as its operands landed,
// each with its own modulus decision (or native fallback); the last block
// runs in C panels, and each panel gets beta C0 added and is written back
// while later panels compute.
int incore_ozaki_kblocks(const Gemm &g, Context *c, DeviceOps &d, int mode, blasx_call_stats &st) {
    Events ev;
    const int blocks = kblock_count(g);
    cudaEvent_t start = ev.make();
    BX_CUDA(cudaEventRecord(start, c->compute));
    BX_CUDA(cudaStreamWaitEvent(c->h2d, start, 0));
    BX_CUDA(cudaStreamWaitEvent(c->d2h, start, 0));
    Gemm dg = g;
    dg.C = d.C;
    dg.ldc = d.ldc;
    OzPanelCtx pctx{&g, &d, c, &ev, &st};
    // each block's compute is enqueued right after its copies: with staged
    // host memory the next block's copies keep this thread busy (packing)
    // while the block computes
    for (int b = 0; b < blocks; ++b) {
        BX_TRY(copy_kblock_in(g, d, kblock_edge(g, b, blocks), kblock_edge(g, b + 1, blocks), c->h2d, st));
        cudaEvent_t in = ev.make();
        BX_CUDA(cudaEventRecord(in, c->h2d));
        BX_CUDA(cudaStreamWaitEvent(c->compute, in, 0));
        Gemm kb = kblock_of(dg, d.A, d.lda, d.B, d.ldb, kblock_edge(g, b, blocks),
                            kblock_edge(g, b + 1, blocks));
        kb.beta = b == 0 ? cplx{0.0, 0.0} : cplx{1.0, 0.0};
        if (b + 1 < blocks) {
            BX_TRY(ozaki_gemm_step(kb, c->compute, mode, d.ws, c->num_sms, b == 0, false));
        } else {
            PanelHooks hooks{panel_count(g), nullptr, &oz_after_panel_kblocks, &pctx};
            BX_TRY(ozaki_gemm_panels(kb, c->compute, mode, d.ws, c->num_sms, hooks, false));
        }
    }
    return finish_ozaki(c, st);
}

int incore_ozaki(const Gemm &g, Context *c, DeviceOps &d, bool read_c, int mode,
                 blasx_call_stats &st) {
    // K-blocks copy A and B in pieces; a stored triangle is completed whole
    if (kblock_count(g) > 1 && !g.a_form && !g.b_form) return incore_ozaki_kblocks(g, c, d, mode, st);
    Events ev;
    const size_t es = elem_size(g.dt);
    cudaEvent_t start = ev.make();
    BX_CUDA(cudaEventRecord(start, c->compute));
    BX_CUDA(cudaStreamWaitEvent(c->h2d, start, 0));
    BX_CUDA(cudaStreamWaitEvent(c->d2h, start, 0));
    // A and B first (the slicing needs them whole); C follows panel by panel,
    // each reconstruction waiting only for its own panel
    BX_TRY(copy2d(d.A, d.lda * es, g.A, g.lda * es, g.rows_a() * es, g.cols_a(),
                              cudaMemcpyHostToDevice, c->h2d));
    if (!d.b_is_a)
        BX_TRY(copy2d(d.B, d.ldb * es, g.B, g.ldb * es, g.rows_b() * es, g.cols_b(),
                                  cudaMemcpyHostToDevice, c->h2d));
    st.h2d_bytes += double(es) * (g.rows_a() * g.cols_a() + (d.b_is_a ? 0 : g.rows_b() * g.cols_b()));
    cudaEvent_t ab = ev.make();
    BX_CUDA(cudaEventRecord(ab, c->h2d));
    BX_CUDA(cudaStreamWaitEvent(c->compute, ab, 0));
    Gemm dg = g;
    dg.A = d.A; dg.lda = d.lda;
    dg.B = d.B; dg.ldb = d.ldb;
    dg.C = d.C; dg.ldc = d.ldc;
    dg.a_form = dg.b_form = 0;
    BX_TRY(complete_forms(g, d, c->compute));
    OzPanelCtx pctx{&g, &d, c, &ev, &st};
    PanelHooks hooks{panel_count(g), read_c ? &oz_before_reconstruct : nullptr, &oz_after_panel,
                     &pctx};
    BX_TRY(ozaki_gemm_panels(dg, c->compute, mode, d.ws, c->num_sms, hooks));
    return finish_ozaki(c, st);
}

bool want_ozaki(const Gemm &g, int mode) { return ozaki_selected(g, mode); }

// Device bytes of host_gemm's in-core path for g: A, B (none when B is A's
// buffer), C, the emulated path's scratch and, when it works in K-blocks
// with C read, the input copy of C.
struct IncoreBytes {
    size_t a = 0, b = 0, c = 0, c0 = 0, ws = 0;
    size_t total() const { return a + b + c + c0 + ws; }
};
IncoreBytes incore_bytes(const Gemm &g, int mode) {
    const size_t es = elem_size(g.dt);
    const bool need_ab = !(g.alpha_zero() || g.K == 0);
    const bool read_c = !g.beta_zero() || g.uplo != 0;
    const bool oz = need_ab && want_ozaki(g, mode);
    const bool shared = need_ab && b_is_a(g);
    IncoreBytes ib;
    ib.a = need_ab ? size_t(round_up(g.rows_a(), 32)) * g.cols_a() * es : 0;
    ib.b = need_ab && !shared ? size_t(round_up(g.rows_b(), 32)) * g.cols_b() * es : 0;
    ib.c = size_t(round_up(g.M, 32)) * g.N * es;
    Gemm probe = g;
    probe.lda = round_up(g.rows_a(), 32);
    probe.ldb = round_up(g.rows_b(), 32);
    probe.ldc = round_up(g.M, 32);
    if (!shared) probe.B = nullptr;  // the scratch shares slices only when the device copy is shared
    probe.a_form = probe.b_form = 0;
    ib.ws = oz ? ozaki_scratch_bytes(probe) : 0;
    ib.c0 = (oz && read_c && kblock_count(g) > 1 && !(g.a_form || g.b_form)) ? ib.c : 0;
    return ib;
}

// The emulated scratch of one tile-cache K-step of g with tile edge T (0
// when the steps run natively).
size_t tile_step_ws(const Gemm &g, int T, int mode) {
    Gemm step = g;
    step.M = std::min<int64_t>(g.M, T);
    step.N = std::min<int64_t>(g.N, T);
    step.K = std::min<int64_t>(g.K, T);
    step.lda = step.ldb = step.ldc = T;
    step.B = nullptr;  // a step's A and B tiles sit in separate slots, even for SYRK
    return want_ozaki(step, mode) ? ozaki_scratch_bytes(step) : 0;
}

// Whether host_gemm runs g under the budget, in core or through the tile
// cache (the C tiles and two operand tiles, and a step's scratch).
bool host_gemm_fits(const Gemm &g, int mode, size_t budget) {
    if (incore_bytes(g, mode).total() <= budget) return true;
    const int T = pick_tile(g, mode, budget);
    return tiled_min_bytes(g.dt, T, tile_step_ws(g, T, mode)) <= budget;
}

}  // namespace

// The blocks of the streamed triangular pipeline: the order K of the
// triangle cut into n blocks of b rows (left) or columns (right), taken in
// substitution order (tri_forward: ascending), the block taken last ragged.
// A solve takes up to 8 blocks of at least 2048, a multiply up to 16 of at
// least 1024 (2 for smaller K): fewer blocks leave longer copies at the
// start and end uncovered, more blocks shrink the update GEMMs (the emulated
// path slices the blocks before each one again). At 16384 these counts
// measured fastest among 4, 6, 8, 12 and 16: a multiply's diagonal blocks
// of 1024 keep their inner updates on the native kernels.
struct TriBlocks {
    int64_t K = 0, b = 0;
    int n = 0;
    bool fwd = true;
    TriBlocks(const Trsm &t, bool mult) : K(t.order()), fwd(tri_forward(t)) {
        const int64_t parts = mult ? std::min<int64_t>(16, std::max<int64_t>(2, K / 1024))
                                   : std::min<int64_t>(8, std::max<int64_t>(2, K / 2048));
        b = round_up((K + parts - 1) / parts, 256);
        n = int((K + b - 1) / b);
    }
    // block i: [lo, hi); the blocks before it: [dlo, dhi) (empty for i == 0)
    void block(int i, int64_t *lo, int64_t *hi, int64_t *dlo, int64_t *dhi) const {
        if (fwd) {
            *lo = i * b;
            *hi = std::min(K, *lo + b);
            *dlo = 0;
            *dhi = *lo;
        } else {
            *hi = K - i * b;
            *lo = std::max<int64_t>(0, *hi - b);
            *dlo = *hi;
            *dhi = K;
        }
    }
};

// TRSM and TRMM with the copies streamed against the compute. Block i of
// the order needs its strip of A (its diagonal block and the rectangle of
// op(A) against the blocks before it, inside the stored triangle) and its
// part of B (rows for a left solve or multiply, columns for a right one);
// the H2D stream copies these block after block, all enqueued at once, the
// compute stream takes each block when its copies landed, and the D2H stream
// returns each block of the result as soon as it is final.
//   solve:    B_i = alpha B_i - op(A)[i, before] X_before (one GEMM), then
//             the solve of block i against its diagonal block;
//   multiply: out of place into R (the earlier blocks' original values are
//             still needed): R_i = alpha S_ii B_i (trmm_part_into), then
//             R_i += alpha op(A)[i, before] B_before (one GEMM).
// The strip is stored as rows i x the blocks up to i (left NoTrans, right
// Trans) or the transpose.
static int tri_streamed(const Trsm &t, const Trsm &dt, const DeviceOps &d, Context *c, bool mult,
                        const TrmmScratch &w, const TriBlocks &tb, bool *emulated, blasx_call_stats &st) {
    const size_t es = elem_size(t.dt);
    Events ev;
    cudaEvent_t start = ev.make();
    BX_CUDA(cudaEventRecord(start, c->compute));  // the device buffers are allocated on compute
    BX_CUDA(cudaStreamWaitEvent(c->h2d, start, 0));
    BX_CUDA(cudaStreamWaitEvent(c->d2h, start, 0));
    // part [p0, p1) of a B-shaped buffer: rows (left) or columns (right)
    auto part = [&](void *base, int64_t ld, int64_t p0) {
        return static_cast<char *>(base) + (t.left ? p0 : p0 * ld) * int64_t(es);
    };
    auto handoff = [&](cudaStream_t from, cudaStream_t to) -> int {
        cudaEvent_t e = ev.make();
        BX_CUDA(cudaEventRecord(e, from));
        BX_CUDA(cudaStreamWaitEvent(to, e, 0));
        return BLASX_OK;
    };
    const bool strip_rows = t.left == (t.trans == NoTrans);
    for (int i = 0; i < tb.n; ++i) {
        int64_t lo, hi, dlo, dhi;
        tb.block(i, &lo, &hi, &dlo, &dhi);
        const int64_t r0 = std::min(lo, dlo), r1 = std::max(hi, dhi);
        const int64_t arow0 = strip_rows ? lo : r0, arow1 = strip_rows ? hi : r1;
        const int64_t acol0 = strip_rows ? r0 : lo, acol1 = strip_rows ? r1 : hi;
        BX_TRY(copy2d(static_cast<char *>(d.A) + (arow0 + acol0 * d.lda) * es, d.lda * es,
                                  static_cast<const char *>(t.A) + (arow0 + acol0 * t.lda) * es, t.lda * es,
                                  (arow1 - arow0) * es, acol1 - acol0, cudaMemcpyHostToDevice, c->h2d));
        const int64_t rows = t.left ? hi - lo : t.M, cols = t.left ? t.N : hi - lo;
        BX_TRY(copy2d(part(d.B, d.ldb, lo), d.ldb * es, part(t.B, t.ldb, lo), t.ldb * es, rows * es, cols,
                                  cudaMemcpyHostToDevice, c->h2d));
        st.h2d_bytes += double(es) * (double(arow1 - arow0) * (acol1 - acol0) + double(rows) * cols);
        BX_TRY(handoff(c->h2d, c->compute));
        if (mult) {
            BX_TRY(trmm_part_into(dt, d.C, lo, hi, w, c->compute, emulated));
            if (dlo < dhi) BX_TRY(trmm_update_into(dt, d.C, lo, hi, dlo, dhi, c->compute, emulated));
        } else if (dlo < dhi) {
            BX_TRY(trsm_update_part(dt, lo, hi, dlo, dhi, t.alpha, c->compute, emulated));
            BX_TRY(trsm_solve_part(dt, lo, hi, cplx{1.0, 0.0}, c->compute, emulated));
        } else {
            BX_TRY(trsm_solve_part(dt, lo, hi, t.alpha, c->compute, emulated));
        }
        BX_TRY(handoff(c->compute, c->d2h));
        BX_TRY(copy2d(part(t.B, t.ldb, lo), t.ldb * es, part(mult ? d.C : d.B, d.ldb, lo), d.ldb * es,
                                  rows * es, cols, cudaMemcpyDeviceToHost, c->d2h));
        st.d2h_bytes += double(es) * rows * cols;
    }
    BX_CUDA(cudaStreamSynchronize(c->h2d));
    BX_CUDA(cudaStreamSynchronize(c->compute));
    BX_CUDA(cudaStreamSynchronize(c->d2h));
    return BLASX_OK;
}

// TRSM / TRMM whose B does not fit the HBM budget beside A: the vectors of B
// (columns for a left solve or multiply, rows for a right one) are
// independent, so B streams through two device panels while A stays
// resident. Panel p + 1 is copied in while panel p computes, and each panel
// goes back as soon as it is done; a panel buffer is refilled only after its
// previous contents left. The panel width is the largest that fits (at least
// 256 vectors; all of B in one panel when only the streamed multiply's
// result buffer did not fit); A itself must fit.
// The device layout of a panel of wv vectors of t (columns for a left call,
// rows for a right one): K x wv (ld K padded) or wv x K (ld wv padded), A
// with ld K padded.
static Trsm tri_panel_desc(const Trsm &t, int64_t wv) {
    const int64_t K = t.order();
    Trsm p = t;
    p.lda = round_up(K, 32);
    if (t.left) { p.N = wv; p.ldb = round_up(K, 32); }
    else { p.M = wv; p.ldb = round_up(wv, 32); }
    return p;
}

// Device bytes of tri_panels with panels of wv vectors: A, two panels, the
// scratch of the largest update GEMM, TRMM's leaf scratch.
static size_t tri_panel_need(const Trsm &t, bool mult, int mode, int64_t wv) {
    const size_t es = elem_size(t.dt);
    const int64_t K = t.order();
    const bool need_a = !(t.alpha.re == 0 && t.alpha.im == 0);  // alpha == 0: B = 0, A and B not read
    const size_t bytes_a = need_a ? size_t(round_up(K, 32)) * K * es : 0;
    const Trsm p = tri_panel_desc(t, wv);
    const Gemm top = mult ? trmm_top_update(p) : trsm_top_update(p);
    const size_t ws = top.K > 0 && ozaki_selected(top, mode) ? ozaki_scratch_bytes(top) : 0;
    const TrmmScratch w = mult ? trmm_scratch_sizes(p) : TrmmScratch{};
    const size_t panel = size_t(p.ldb) * size_t(t.left ? wv : K) * es;
    return bytes_a + 2 * panel + ws + w.diag_bytes + w.temp_bytes;
}

static int tri_panels(const Trsm &t, Context *c, bool mult, int mode, size_t budget, blasx_call_stats &st) {
    const size_t es = elem_size(t.dt);
    const int64_t K = t.order(), nvec = t.left ? t.N : t.M;
    const int64_t lda = round_up(K, 32);
    const bool need_a = !(t.alpha.re == 0 && t.alpha.im == 0);  // alpha == 0: B = 0, A and B not read
    const size_t bytes_a = need_a ? size_t(lda) * K * es : 0;
    auto panel_desc = [&](int64_t wv) { return tri_panel_desc(t, wv); };
    auto need = [&](int64_t wv) { return tri_panel_need(t, mult, mode, wv); };
    int64_t wv = nvec;
    while (wv > 256 && need(wv) > budget) wv = (wv / 2 + 31) / 32 * 32;
    if (need(wv) > budget)
        return set_error(BLASX_ERR_UNSUPPORTED, "triangular %s: A (%zu bytes) leaves no room for panels of B in "
                         "the HBM budget", mult ? "multiply" : "solve", bytes_a);
    const Trsm full = panel_desc(wv);
    const size_t panel_bytes = size_t(full.ldb) * size_t(t.left ? wv : K) * es;
    TrmmScratch w = mult ? trmm_scratch_sizes(full) : TrmmScratch{};
    HostPin pins;
    BX_TRY(pins.pin(t.A, need_a ? host_extent(t.lda, K, K, es) : 0));
    BX_TRY(pins.pin(t.B, host_extent(t.ldb, t.M, t.N, es)));
    st.host_copy = pins.mode();
    DeviceOps d;
    d.s = c->compute;
    StreamDrain drain{c};  // before d and pins go, on every return
    if (need_a) BX_CUDA(dev_malloc_async(&d.A, bytes_a, c->compute));
    BX_CUDA(dev_malloc_async(&d.B, 2 * panel_bytes, c->compute));
    if (mult && need_a) {
        BX_CUDA(dev_malloc_async(&d.diag, w.diag_bytes, c->compute));
        BX_CUDA(dev_malloc_async(&d.C0, w.temp_bytes, c->compute));
        w.diag = d.diag;
        w.temp = d.C0;
    }
    Events ev;
    auto handoff = [&](cudaStream_t from, cudaStream_t to) -> int {
        cudaEvent_t e = ev.make();
        BX_CUDA(cudaEventRecord(e, from));
        BX_CUDA(cudaStreamWaitEvent(to, e, 0));
        return BLASX_OK;
    };
    BX_TRY(handoff(c->compute, c->h2d));  // the buffers are allocated on compute
    if (need_a) {
        BX_TRY(copy2d(d.A, lda * es, t.A, t.lda * es, K * es, K, cudaMemcpyHostToDevice, c->h2d));
        st.h2d_bytes += double(es) * K * K;
    }
    cudaEvent_t out_done[2] = {nullptr, nullptr};
    bool emulated = false;
    for (int64_t v0 = 0, p = 0; v0 < nvec; v0 += wv, ++p) {
        const int64_t v1 = std::min(nvec, v0 + wv), n = v1 - v0;
        const int buf = int(p & 1);
        Trsm tp = panel_desc(n);
        tp.A = d.A;
        tp.B = static_cast<char *>(d.B) + buf * panel_bytes;
        tp.ldb = full.ldb;
        char *host = static_cast<char *>(t.B) + (t.left ? v0 * t.ldb : v0) * int64_t(es);
        const int64_t rows = t.left ? t.M : n, cols = t.left ? n : t.N;
        if (out_done[buf]) BX_CUDA(cudaStreamWaitEvent(c->h2d, out_done[buf], 0));
        if (need_a) {
            BX_TRY(copy2d(tp.B, tp.ldb * es, host, t.ldb * es, rows * es, cols, cudaMemcpyHostToDevice,
                                      c->h2d));
            st.h2d_bytes += double(es) * rows * cols;
        }
        BX_TRY(handoff(c->h2d, c->compute));
        bool e = false;
        BX_TRY(mult ? trmm_device(tp, w, c->compute, &e) : trsm_device(tp, c->compute, &e));
        emulated |= e;
        BX_TRY(handoff(c->compute, c->d2h));
        BX_TRY(copy2d(host, t.ldb * es, tp.B, tp.ldb * es, rows * es, cols, cudaMemcpyDeviceToHost,
                                  c->d2h));
        st.d2h_bytes += double(es) * rows * cols;
        if (!out_done[buf]) out_done[buf] = ev.make();
        BX_CUDA(cudaEventRecord(out_done[buf], c->d2h));
    }
    BX_CUDA(cudaStreamSynchronize(c->h2d));
    BX_CUDA(cudaStreamSynchronize(c->compute));
    BX_CUDA(cudaStreamSynchronize(c->d2h));
    BX_TRY(pins.finish());  // staged write-backs in host memory
    st.path = !need_a ? 3 : (emulated ? 2 : 1);
    st.tile = int(wv);  // the panel width, in vectors
    if (emulated) {
        resolve_decision(st);
        if (*c->last_error_flag)
            return set_error(BLASX_ERR_TIMEOUT, "emulated GEMM: bounded device wait expired (flag %d)",
                             *c->last_error_flag);
    }
    return BLASX_OK;
}

// TRSM (mult false) or TRMM (mult true) on host operands: A (the order-K
// triangle) and B to the device, the solve or multiply, B back. A triangle
// of more than one block streams its copies against the compute block by
// block (tri_streamed); one block is copied, solved or multiplied by the
// recursion, and copied back. The scratch of the largest update GEMM (and
// TRMM's leaf scratch and result buffer) is part of the budget; a B beyond
// it streams in panels (tri_panels).
static int host_tri(const Trsm &t, bool mult) {
    auto t0 = std::chrono::steady_clock::now();
    blasx_call_stats &st = call_stats();
    st = blasx_call_stats{};
    if (t.M == 0 || t.N == 0) return BLASX_OK;
    Context *c = context();
    if (!c) return last_status();
    std::lock_guard<std::mutex> lk(c->host_mu);
    const int mode = config().dgemm_mode.load();
    const size_t es = elem_size(t.dt);
    const int64_t K = t.order();
    const bool need_a = !(t.alpha.re == 0 && t.alpha.im == 0);
    DeviceOps d;
    d.s = c->compute;
    d.lda = round_up(K, 32);
    d.ldb = round_up(t.M, 32);
    Trsm dt = t;
    dt.lda = d.lda;
    dt.ldb = d.ldb;
    const size_t bytes_a = need_a ? size_t(d.lda) * K * es : 0;
    const size_t bytes_b = size_t(d.ldb) * t.N * es;
    auto ws_of = [&](const Gemm &g) { return g.K > 0 && ozaki_selected(g, mode) ? ozaki_scratch_bytes(g) : size_t(0); };
    const TriBlocks tb(dt, mult);
    const bool split = need_a && tb.n > 1;
    size_t bytes_ws = 0, bytes_r = 0;
    if (need_a) {
        Trsm blk = dt;  // the recursion inside one block (the whole triangle unsplit)
        if (split) (t.left ? blk.M : blk.N) = tb.b;
        bytes_ws = ws_of(mult ? trmm_top_update(blk) : trsm_top_update(blk));
        if (split) {  // the largest block update: the last block's, from all the others
            int64_t lo, hi, dlo, dhi;
            tb.block(tb.n - 1, &lo, &hi, &dlo, &dhi);
            bytes_ws = std::max(bytes_ws, ws_of(tri_update_gemm(dt, lo, hi, dlo, dhi)));
            if (mult) bytes_r = bytes_b;  // the out-of-place result
        }
    }
    TrmmScratch w = mult ? trmm_scratch_sizes(dt) : TrmmScratch{};
    const size_t bytes_w = need_a ? w.diag_bytes + w.temp_bytes : 0;
    const size_t budget = default_budget(c);
    if (bytes_a + bytes_b + bytes_r + bytes_ws + bytes_w > budget) {
        const int rc = tri_panels(t, c, mult, mode, budget, st);
        st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return rc;
    }
    HostPin pins;
    BX_TRY(pins.pin(t.A, need_a ? host_extent(t.lda, K, K, es) : 0));
    BX_TRY(pins.pin(t.B, host_extent(t.ldb, t.M, t.N, es)));
    st.host_copy = pins.mode();
    StreamDrain drain{c};  // before d and pins go, on every return
    cudaStream_t s = c->compute;
    if (need_a) BX_CUDA(dev_malloc_async(&d.A, bytes_a, s));
    BX_CUDA(dev_malloc_async(&d.B, bytes_b, s));  // alpha == 0 writes zeros without reading B
    if (bytes_r) BX_CUDA(dev_malloc_async(&d.C, bytes_r, s));
    if (bytes_w) {
        BX_CUDA(dev_malloc_async(&d.diag, w.diag_bytes, s));
        BX_CUDA(dev_malloc_async(&d.C0, w.temp_bytes, s));
        w.diag = d.diag;
        w.temp = d.C0;
    }
    dt.A = d.A;
    dt.B = d.B;
    bool emulated = false;
    if (!split) {
        if (need_a) {
            BX_TRY(copy2d(d.A, d.lda * es, t.A, t.lda * es, K * es, K, cudaMemcpyHostToDevice, s));
            BX_TRY(copy2d(d.B, d.ldb * es, t.B, t.ldb * es, t.M * es, t.N, cudaMemcpyHostToDevice, s));
            st.h2d_bytes += double(es) * (double(K) * K + double(t.M) * t.N);
        }
        BX_TRY(mult ? trmm_device(dt, w, s, &emulated) : trsm_device(dt, s, &emulated));
        BX_TRY(copy2d(t.B, t.ldb * es, d.B, d.ldb * es, t.M * es, t.N, cudaMemcpyDeviceToHost, s));
        st.d2h_bytes += double(es) * t.M * t.N;
        BX_CUDA(cudaStreamSynchronize(s));
    } else {
        BX_TRY(tri_streamed(t, dt, d, c, mult, w, tb, &emulated, st));
        st.tile = int(tb.b);  // the block order
    }
    BX_TRY(pins.finish());  // staged write-backs in host memory
    st.path = !need_a ? 3 : (emulated ? 2 : 1);
    if (emulated) {
        resolve_decision(st);
        if (*c->last_error_flag)
            return set_error(BLASX_ERR_TIMEOUT, "emulated GEMM: bounded device wait expired (flag %d)",
                             *c->last_error_flag);
    }
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return BLASX_OK;
}

namespace {

// ---- an A beyond the budget: the order halved on the host ---------------
// When A leaves no room for panels of B, the order is halved on the host as
// the device recursion halves it: each diagonal half is a solve or multiply
// of its own (halved again until its A fits), on the host operands at an
// offset, and the off-diagonal block is one host GEMM, through the tile
// cache when it does not fit in core.
//   solve:    solve(first, alpha); B_second = alpha B_second - op(A)[second, first] X_first;
//             solve(second, 1)
//   multiply: multiply(first); B_first += alpha op(A)[first, second] B_second (its
//             original values); multiply(second)
// with first the earlier half in substitution order for the solve, the later
// one for the multiply.

bool tri_fits(const Trsm &t, bool mult, int mode, size_t budget) {
    const int64_t nvec = t.left ? t.N : t.M;
    return tri_panel_need(t, mult, mode, std::min<int64_t>(nvec, 256)) <= budget;
}

// the split point of a host halving: the earlier part has m rows
int64_t host_half(int64_t K) { return std::min(K - 1, round_up((K + 1) / 2, 256)); }

// t with its order restricted to [lo, hi): A's diagonal block, B's rows
// (left) or columns (right)
Trsm tri_piece(const Trsm &t, int64_t lo, int64_t hi, cplx alpha) {
    const size_t es = elem_size(t.dt);
    Trsm p = t;
    p.A = static_cast<const char *>(t.A) + (lo + lo * t.lda) * int64_t(es);
    p.B = static_cast<char *>(t.B) + (t.left ? lo : lo * t.ldb) * int64_t(es);
    (t.left ? p.M : p.N) = hi - lo;
    p.alpha = alpha;
    return p;
}

void merge_stats(blasx_call_stats &agg, const blasx_call_stats &s) {
    agg.h2d_bytes += s.h2d_bytes;
    agg.d2h_bytes += s.d2h_bytes;
    agg.cache_hits += s.cache_hits;
    agg.cache_misses += s.cache_misses;
    agg.evictions += s.evictions;
    auto rank = [](int p) { return p == 2 ? 3 : p == 4 ? 2 : p == 1 ? 1 : 0; };
    if (rank(s.path) > rank(agg.path)) agg.path = s.path;
    if (s.path == 2) agg.moduli = std::max(agg.moduli, s.moduli);
}

int tri_split(const Trsm &t, bool mult, int mode, size_t budget, blasx_call_stats &agg);

int tri_run(const Trsm &t, bool mult, int mode, size_t budget, blasx_call_stats &agg) {
    if (!tri_fits(t, mult, mode, budget)) return tri_split(t, mult, mode, budget, agg);
    const int rc = host_tri(t, mult);
    merge_stats(agg, call_stats());
    agg.tile = std::max<int>(agg.tile, int(t.order()));
    return rc;
}

// The halves of a host halving, in the order they run: first [f0, f1),
// then second [s0, s1); the lower part is [0, m), the upper [m, K).
struct TriHalves {
    int64_t f0, f1, s0, s1;
    TriHalves(const Trsm &t, bool mult) {
        const int64_t K = t.order(), m = host_half(K);
        const bool fwd = tri_forward(t);
        const bool lower_first = mult ? !fwd : fwd;
        f0 = lower_first ? 0 : m; f1 = lower_first ? m : K;
        s0 = lower_first ? m : 0; s1 = lower_first ? K : m;
    }
    // the off-diagonal update: the second half from the first (solve), or
    // the first from the second (multiply); alpha and beta as tri_split sets them
    Gemm update(const Trsm &t, bool mult) const {
        if (mult) return tri_update_gemm(t, f0, f1, s0, s1);
        Gemm g = tri_update_gemm(t, s0, s1, f0, f1);
        g.alpha = cplx{-1.0, 0.0};
        g.beta = t.alpha;
        return g;
    }
};

int tri_split(const Trsm &t, bool mult, int mode, size_t budget, blasx_call_stats &agg) {
    const TriHalves h(t, mult);
    const int64_t f0 = h.f0, f1 = h.f1, s0 = h.s0, s1 = h.s1;
    if (mult) {
        BX_TRY(tri_run(tri_piece(t, f0, f1, t.alpha), true, mode, budget, agg));
        BX_TRY(host_gemm(h.update(t, true)));
        merge_stats(agg, call_stats());
        return tri_run(tri_piece(t, s0, s1, t.alpha), true, mode, budget, agg);
    }
    BX_TRY(tri_run(tri_piece(t, f0, f1, t.alpha), false, mode, budget, agg));
    BX_TRY(host_gemm(h.update(t, false)));
    merge_stats(agg, call_stats());
    return tri_run(tri_piece(t, s0, s1, cplx{1.0, 0.0}), false, mode, budget, agg);
}

// TRSM / TRMM on host operands: one host_tri call, or the host halving when
// A does not fit. The halving is checked whole before it starts (every
// piece fits at the depth it reaches, and the largest update GEMM can run),
// so that a call the budget cannot hold leaves B unchanged.
int host_tri_entry(const Trsm &t, bool mult) {
    const bool need_a = !(t.alpha.re == 0 && t.alpha.im == 0);
    if (t.M == 0 || t.N == 0 || !need_a) return host_tri(t, mult);
    Context *c = context();
    if (!c) {
        call_stats() = blasx_call_stats{};
        return last_status();
    }
    const int mode = config().dgemm_mode.load();
    const size_t budget = default_budget(c);
    if (tri_fits(t, mult, mode, budget)) return host_tri(t, mult);
    auto t0 = std::chrono::steady_clock::now();
    call_stats() = blasx_call_stats{};
    const int64_t K = t.order();
    int64_t o = K;
    while (o > 256 && !tri_fits(tri_piece(t, 0, o, t.alpha), mult, mode, budget)) o = std::max(host_half(o), o - host_half(o));
    if (!tri_fits(tri_piece(t, 0, o, t.alpha), mult, mode, budget))
        return set_error(BLASX_ERR_UNSUPPORTED, "triangular %s: the HBM budget (%zu bytes) holds no piece of A "
                         "with room for panels of B", mult ? "multiply" : "solve", budget);
    const Gemm top = TriHalves(t, mult).update(t, mult);  // the largest update
    if (!host_gemm_fits(top, mode, budget))
        return set_error(BLASX_ERR_UNSUPPORTED, "triangular %s: the HBM budget (%zu bytes) cannot hold the "
                         "update GEMM of its halves (tile edge %d)", mult ? "multiply" : "solve", budget,
                         pick_tile(top, mode, budget));
    // registered once for every part (the parts' own registrations would
    // overlap); staged ranges are staged again by each part's own call
    HostPin pins;
    const size_t es = elem_size(t.dt);
    BX_TRY(pins.pin(t.A, host_extent(t.lda, K, K, es)));
    BX_TRY(pins.pin(t.B, host_extent(t.ldb, t.M, t.N, es)));
    blasx_call_stats agg{};
    agg.host_copy = pins.mode();
    const int rc = tri_split(t, mult, mode, budget, agg);
    agg.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    call_stats() = agg;
    return rc;
}

}  // namespace

int host_trsm(const Trsm &t) { return host_tri_entry(t, false); }
int host_trmm(const Trsm &t) { return host_tri_entry(t, true); }

int host_gemm(const Gemm &g) {
    auto t0 = std::chrono::steady_clock::now();
    blasx_call_stats &st = call_stats();
    st = blasx_call_stats{};
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    Context *c = context();
    if (!c) return last_status();
    std::lock_guard<std::mutex> lk(c->host_mu);
    const size_t es = elem_size(g.dt);
    const bool need_ab = !(g.alpha_zero() || g.K == 0);
    // a triangular output keeps the other triangle: C always makes the round trip
    const bool read_c = !g.beta_zero() || g.uplo != 0;
    const int mode = config().dgemm_mode.load();
    const bool oz = need_ab && want_ozaki(g, mode);

    DeviceOps d;
    d.s = c->compute;
    d.b_is_a = need_ab && b_is_a(g);
    d.lda = round_up(g.rows_a(), 32);
    d.ldb = round_up(g.rows_b(), 32);
    d.ldc = round_up(g.M, 32);
    const IncoreBytes ib = incore_bytes(g, mode);
    const size_t budget = default_budget(c);

    HostPin pins;
    // out of core, a symmetric / Hermitian operand (SYMM, HEMM) is read tile by
    // tile from its stored triangle (tiled_host_gemm)
    if (ib.total() > budget && need_ab) {
        // out-of-core: HBM tile cache under the byte budget; each K-step on
        // the emulated path when the precision mode picks it for a step's shape
        const int T = pick_tile(g, mode, budget);
        const int st_code = tiled_host_gemm(g, c, budget, T, 0, tile_step_ws(g, T, mode), mode);
        st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return st_code;
    }
    BX_TRY(pins.pin(g.A, need_ab ? host_extent(g.lda, g.rows_a(), g.cols_a(), es) : 0));
    BX_TRY(pins.pin(g.B, need_ab && !d.b_is_a ? host_extent(g.ldb, g.rows_b(), g.cols_b(), es) : 0));
    BX_TRY(pins.pin(g.C, host_extent(g.ldc, g.M, g.N, es)));
    st.host_copy = pins.mode();
    StreamDrain drain{c};  // before d and pins go, on every return
    if (need_ab) {
        BX_CUDA(dev_malloc_async(&d.A, ib.a ? ib.a : 256, c->compute));
        if (d.b_is_a) d.B = d.A;
        else BX_CUDA(dev_malloc_async(&d.B, ib.b ? ib.b : 256, c->compute));
    }
    BX_CUDA(dev_malloc_async(&d.C, ib.c, c->compute));
    if (oz) BX_CUDA(dev_malloc_async(&d.ws, ib.ws, c->compute));
    if (ib.c0) BX_CUDA(dev_malloc_async(&d.C0, ib.c0, c->compute));
    int rc = oz ? incore_ozaki(g, c, d, read_c, mode, st)
                : incore_native(g, c, d, need_ab, read_c, st);
    if (rc == BLASX_OK) rc = pins.finish();  // staged write-backs in host memory
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

}  // namespace bx
