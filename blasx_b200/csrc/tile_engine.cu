// tile_engine.cu -- executes a TilePlan for a host GEMM larger than the HBM
// budget (out-of-core), on the native kernels or, K-step by K-step, on the
// emulated (Ozaki) path.
//
// Replaces the reference's worker loop (blas/blasx_dgemm.c:98-248: batches
// of 4 tasks, a host busy-wait on an event, cudaStreamSynchronize after the
// copies of every tile-step, serial write-back of C) with a plan enqueued in
// one pass over three streams, ordered only by events:
//   H2D stream      operand tile -> its slot; C tile -> a C slot (beta != 0);
//                   a reload into a slot first waits for the slot's last use;
//   compute stream  waits for the tile's ready event, runs the K-step GEMM
//                   (beta on the first K-step, 1 afterwards as in
//                   blas/blasx_dgemm.c:82), records the slot's last use;
//                   an emulated K-step slices both tiles, runs the residue
//                   GEMMs and adds alpha X into the C tile in FP64, with its
//                   own modulus decision (native fallback on the device);
//   D2H stream      writes a finished C tile back to the host.
// With pinned host operands the host thread never blocks until the final
// synchronisation, so copies run ahead of compute as far as slot reuse
// allows. Pageable host operands are staged through pinned bounce buffers
// (staging.h): the host thread then packs each inbound tile and waits for
// outbound buffers, which keeps the copies about one C tile ahead. With
// staging switched off they are registered for the duration of the call over
// their full ld x columns extent (the reference registers rows x columns,
// blas/dgemm.c:88-90, which misses the ld padding).
#include <chrono>
#include <mutex>
#include <vector>

#include "kernels.h"
#include "ozaki.h"
#include "tile_engine.h"
#include "tile_plan.h"

namespace bx {

namespace {

constexpr int kCSlots = kCTileSlots;

std::mutex g_arena_mu;
void *g_arena = nullptr;
size_t g_arena_bytes = 0;

int ensure_arena(size_t bytes) {
    if (g_arena && g_arena_bytes >= bytes) return BLASX_OK;
    if (g_arena) {
        cudaFree(g_arena);
        g_arena = nullptr;
        g_arena_bytes = 0;
    }
    BX_CUDA(dev_malloc(&g_arena, bytes));
    g_arena_bytes = bytes;
    return BLASX_OK;
}

struct EventPool {
    std::vector<cudaEvent_t> evs;
    ~EventPool() {
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
    }
    int make(cudaEvent_t *out) {
        BX_CUDA(cudaEventCreateWithFlags(out, cudaEventDisableTiming));
        evs.push_back(*out);
        return BLASX_OK;
    }
};

}  // namespace

size_t host_extent(int64_t ld, int64_t rows, int64_t cols, size_t es) {
    if (rows <= 0 || cols <= 0) return 0;
    return (size_t(ld) * size_t(cols - 1) + size_t(rows)) * es;
}

size_t tiled_min_bytes(DType dt, int T, size_t ws_bytes) {
    const size_t ws_reserve = ws_bytes ? ((ws_bytes + 255) & ~size_t(255)) + 256 : 0;
    return size_t(kCSlots + 2) * size_t(T) * T * elem_size(dt) + ws_reserve;
}

int tiled_host_gemm(const Gemm &g, Context *c, size_t budget, int T, int policy, size_t ws_bytes,
                    int mode) {
    blasx_call_stats &st = call_stats();
    const size_t es = elem_size(g.dt);
    const size_t slot_bytes = size_t(T) * T * es;
    const size_t ws_reserve = ws_bytes ? ((ws_bytes + 255) & ~size_t(255)) + 256 : 0;
    const int64_t total_slots = int64_t((budget > ws_reserve ? budget - ws_reserve : 0) / slot_bytes);
    const int op_slots = int(total_slots - kCSlots);
    if (op_slots < 2)
        return set_error(BLASX_ERR_NOMEM, "HBM budget %zu B holds fewer than %d tiles of %d^2",
                         budget, kCSlots + 2, T);
    TilePlan plan;
    if (!plan_tiles(g.M, g.N, g.K, T, op_slots, policy, &plan))
        return set_error(BLASX_ERR_ARG, "tile plan failed");
    {
        std::lock_guard<std::mutex> lk(g_arena_mu);
        BX_TRY(ensure_arena(size_t(op_slots + kCSlots) * slot_bytes + ws_reserve));
    }
    char *arena = static_cast<char *>(g_arena);
    auto op_ptr = [&](int s) { return arena + size_t(s) * slot_bytes; };
    auto c_ptr = [&](int s) { return arena + size_t(op_slots + s) * slot_bytes; };
    // emulated K-steps: scratch after the C slots, 256-byte aligned
    void *ws = nullptr;
    if (ws_bytes) {
        const size_t off = (size_t(op_slots + kCSlots) * slot_bytes + 255) & ~size_t(255);
        ws = arena + off;
    }

    HostPin pins;
    BX_TRY(pins.pin(g.A, host_extent(g.lda, g.rows_a(), g.cols_a(), es)));
    BX_TRY(pins.pin(g.B, host_extent(g.ldb, g.rows_b(), g.cols_b(), es)));
    BX_TRY(pins.pin(g.C, host_extent(g.ldc, g.M, g.N, es)));
    st.host_copy = pins.mode();
    StreamDrain drain{c};  // before pins go, on every return

    EventPool pool;
    std::vector<cudaEvent_t> ready(static_cast<size_t>(op_slots)), lastuse(static_cast<size_t>(op_slots));
    std::vector<bool> used(static_cast<size_t>(op_slots), false);
    cudaEvent_t c_ready[kCSlots], c_done[kCSlots], c_out[kCSlots];
    bool c_used[kCSlots] = {false, false, false};
    for (int s = 0; s < op_slots; ++s) {
        BX_TRY(pool.make(&ready[size_t(s)]));
        BX_TRY(pool.make(&lastuse[size_t(s)]));
    }
    for (int s = 0; s < kCSlots; ++s) {
        BX_TRY(pool.make(&c_ready[s]));
        BX_TRY(pool.make(&c_done[s]));
        BX_TRY(pool.make(&c_out[s]));
    }
    cudaEvent_t start_ev;
    BX_TRY(pool.make(&start_ev));
    BX_CUDA(cudaEventRecord(start_ev, c->compute));
    BX_CUDA(cudaStreamWaitEvent(c->h2d, start_ev, 0));
    BX_CUDA(cudaStreamWaitEvent(c->d2h, start_ev, 0));

    auto ext = [&](int idx, int64_t n) { return std::min<int64_t>(T, n - int64_t(idx) * T); };
    const char *hA = static_cast<const char *>(g.A);
    const char *hB = static_cast<const char *>(g.B);
    char *hC = static_cast<char *>(g.C);

    // A symmetric / Hermitian operand stored as one triangle (SYMM, HEMM; its
    // op is NoTrans): a tile of its stored triangle loads as it is; a tile
    // of the other triangle is the (conjugate) transpose of the stored tile
    // across the diagonal, which loads in its place and multiplies with a
    // transposed op; a diagonal tile is completed in place once it lands.
    auto form_of = [&](int op) { return op == 0 ? g.a_form : g.b_form; };
    enum { kStored = 0, kMirrored = 1, kDiagonal = 2 };
    auto tile_kind = [&](int op, int r, int col) {
        const int f = form_of(op);
        if (!f) return int(kStored);
        if (r == col) return int(kDiagonal);
        const bool upper = f == kSymUpper || f == kHermUpper;
        return (r < col) == upper ? int(kStored) : int(kMirrored);
    };
    auto mirrored_op = [&](int op) {
        const int f = form_of(op);
        return (f == kHermUpper || f == kHermLower) ? int(ConjT) : int(TransT);
    };

    // host address and extent of an operand tile (stored layout)
    auto load_tile = [&](const TileUse &u, const TileStep &s) -> int {
        const bool isA = u.key.op == 0;
        const int64_t rows_op = isA ? ext(s.i, g.M) : ext(s.k, g.K);  // op() rows
        const int64_t cols_op = isA ? ext(s.k, g.K) : ext(s.j, g.N);
        const int64_t r0 = int64_t(isA ? s.i : s.k) * T, c0 = int64_t(isA ? s.k : s.j) * T;
        const int kind = tile_kind(u.key.op, isA ? s.i : s.k, isA ? s.k : s.j);
        // a mirrored tile copies the stored block across the diagonal, as a transposed op would
        const bool tr = kind == kMirrored || (isA ? g.ta != NoTrans : g.tb != NoTrans);
        const int64_t srow = tr ? c0 : r0, scol = tr ? r0 : c0;
        const int64_t nrow = tr ? cols_op : rows_op, ncol = tr ? rows_op : cols_op;
        const int64_t ld = isA ? g.lda : g.ldb;
        const char *src = (isA ? hA : hB) + (srow + scol * ld) * int64_t(es);
        if (used[size_t(u.slot)]) BX_CUDA(cudaStreamWaitEvent(c->h2d, lastuse[size_t(u.slot)], 0));
        BX_TRY(copy2d(op_ptr(u.slot), size_t(T) * es, src, size_t(ld) * es,
                                  size_t(nrow) * es, size_t(ncol), cudaMemcpyHostToDevice, c->h2d));
        if (kind == kDiagonal)
            BX_TRY(launch_complete_operand(g.dt, form_of(u.key.op), op_ptr(u.slot), T, rows_op, c->h2d));
        BX_CUDA(cudaEventRecord(ready[size_t(u.slot)], c->h2d));
        st.h2d_bytes += double(nrow) * ncol * es;
        return BLASX_OK;
    };

    // triangular output: C tiles with no entry inside the triangle are
    // skipped (no C copies, no compute); the others compute with the
    // diagonal shifted to the tile's origin
    auto c_needed = [&](const TileStep &s) {
        if (g.uplo == 0) return true;
        const int64_t i0 = int64_t(s.i) * T, j0 = int64_t(s.j) * T;
        const int64_t m = ext(s.i, g.M), n = ext(s.j, g.N);
        return g.uplo == 1 ? i0 - (j0 + n - 1) <= g.diag : (i0 + m - 1) - j0 >= g.diag;
    };
    size_t last_needed = 0;
    for (size_t i = 0; i < plan.steps.size(); ++i)
        if (c_needed(plan.steps[i])) last_needed = i + 1;
    int ctile = -1;
    size_t step_no = 0;
    bool first_emulated = true;
    for (const TileStep &s : plan.steps) {
        ++step_no;
        if (s.a.load) BX_TRY(load_tile(s.a, s));
        if (s.b.load) BX_TRY(load_tile(s.b, s));
        const int64_t m = ext(s.i, g.M), n = ext(s.j, g.N), k = ext(s.k, g.K);
        const bool needed = c_needed(s);
        if (s.first_k) ++ctile;
        if (!needed) continue;
        if (s.first_k) {
            const int cs = ctile % kCSlots;
            if (c_used[cs]) {  // previous occupant written back before reuse
                BX_CUDA(cudaStreamWaitEvent(c->h2d, c_out[cs], 0));
                BX_CUDA(cudaStreamWaitEvent(c->compute, c_out[cs], 0));
            }
            c_used[cs] = true;
            if (!g.beta_zero() || g.uplo != 0) {  // a triangular tile keeps its other entries
                char *src = hC + (int64_t(s.i) * T + int64_t(s.j) * T * g.ldc) * int64_t(es);
                BX_TRY(copy2d(c_ptr(cs), size_t(T) * es, src, size_t(g.ldc) * es,
                                          size_t(m) * es, size_t(n), cudaMemcpyHostToDevice, c->h2d));
                BX_CUDA(cudaEventRecord(c_ready[cs], c->h2d));
                BX_CUDA(cudaStreamWaitEvent(c->compute, c_ready[cs], 0));
                st.h2d_bytes += double(m) * n * es;
            }
        }
        const int cs = ctile % kCSlots;
        BX_CUDA(cudaStreamWaitEvent(c->compute, ready[size_t(s.a.slot)], 0));
        BX_CUDA(cudaStreamWaitEvent(c->compute, ready[size_t(s.b.slot)], 0));
        Gemm d = g;
        d.M = m; d.N = n; d.K = k;
        d.A = op_ptr(s.a.slot); d.lda = T;
        d.B = op_ptr(s.b.slot); d.ldb = T;
        if (tile_kind(0, s.i, s.k) == kMirrored) d.ta = mirrored_op(0);
        if (tile_kind(1, s.k, s.j) == kMirrored) d.tb = mirrored_op(1);
        d.a_form = d.b_form = 0;
        d.C = c_ptr(cs); d.ldc = T;
        if (!s.first_k) d.beta = cplx{1.0, 0.0};
        d.guard = nullptr;
        d.diag = g.diag + (int64_t(s.j) - int64_t(s.i)) * T;
        if (ws) {
            BX_TRY(ozaki_gemm_step(d, c->compute, mode, ws, c->num_sms, first_emulated,
                                   step_no == last_needed));
            first_emulated = false;
        } else
            BX_TRY(dmma_supported(d) ? launch_gemm_dmma(d, c->compute) : launch_gemm_simt(d, c->compute));
        BX_CUDA(cudaEventRecord(lastuse[size_t(s.a.slot)], c->compute));
        BX_CUDA(cudaEventRecord(lastuse[size_t(s.b.slot)], c->compute));
        used[size_t(s.a.slot)] = used[size_t(s.b.slot)] = true;
        if (s.last_k) {
            if (g.herm_out)  // the global diagonal (row - col == diag) in this tile's coordinates
                BX_TRY(launch_real_diagonal(g.dt, c_ptr(cs), T, m, n, d.diag, c->compute));
            BX_CUDA(cudaEventRecord(c_done[cs], c->compute));
            BX_CUDA(cudaStreamWaitEvent(c->d2h, c_done[cs], 0));
            char *dst = hC + (int64_t(s.i) * T + int64_t(s.j) * T * g.ldc) * int64_t(es);
            BX_TRY(copy2d(dst, size_t(g.ldc) * es, c_ptr(cs), size_t(T) * es,
                                      size_t(m) * es, size_t(n), cudaMemcpyDeviceToHost, c->d2h));
            BX_CUDA(cudaEventRecord(c_out[cs], c->d2h));
            st.d2h_bytes += double(m) * n * es;
        }
    }
    BX_CUDA(cudaStreamSynchronize(c->h2d));
    BX_CUDA(cudaStreamSynchronize(c->compute));
    BX_CUDA(cudaStreamSynchronize(c->d2h));
    BX_TRY(pins.finish());  // staged write-backs in host memory
    st.cache_hits = double(plan.hits);
    st.cache_misses = double(plan.loads);
    st.evictions = double(plan.evictions);
    st.tile = T;
    st.path = ws ? 2 : 1;
    if (ws) {
        resolve_decision(st);  // the last K-step's modulus count
        if (*c->last_error_flag)
            return set_error(BLASX_ERR_TIMEOUT, "emulated tile step: bounded device wait expired (flag %d)",
                             *c->last_error_flag);
    }
    return BLASX_OK;
}

void release_tile_arena() {
    std::lock_guard<std::mutex> lk(g_arena_mu);
    if (g_arena) cudaFree(g_arena);
    g_arena = nullptr;
    g_arena_bytes = 0;
}

}  // namespace bx
