// serving.cu -- continuous batching of host GEMM calls from many threads.
//
// When the serving loop runs (blasx_serve_start), cblas_?gemm / ?gemm_ calls
// from any number of host threads become requests in one queue, served by a
// single scheduler thread that owns the device:
//
//   admission   in arrival order; a request is admitted when an in-flight slot
//               is free and its device bytes (A, B, C copies and the emulated
//               path's scratch) fit the HBM budget; a B operand found in the
//               operand cache is not copied again and not charged again.
//               Requests behind one that waits for memory may pass it if they
//               fit, until it has waited 50 ms (then its memory is kept free);
//   in flight   every admitted request gets its own stream for its copies in
//               and out, which overlap with other requests' compute, and
//               requests that arrive meanwhile are admitted as slots and
//               memory free up;
//   mixing      one persistent kernel (executor.cu) runs the work of every
//               request in flight: native FP64 / complex128 DMMA tiles, FP32 /
//               complex64 SIMT tiles, and each stage of emulated requests
//               (statistics, decision, slices, tcgen05 residue tiles,
//               reconstruction). The scheduler publishes a request's stage
//               into the executor's task ring once its copies (or its
//               previous stage) completed; the kernel's CTAs claim tasks of
//               all requests in publication order, so their tiles share the
//               SMs. Requests whose operand is stored as one triangle (SYMM,
//               HEMM) or whose output is Hermitian run on their own kernels,
//               alone, with the executor stopped;
//   completion  detected by polling each request's last event; device memory
//               is released, the B copy is kept in the operand cache (LRU,
//               byte budget, pinned while in use) and the caller wakes up.
//
// Operand-cache identity rule: a cached device copy of B is reused when the
// host pointer, leading dimension, stored shape and dtype match AND a
// fingerprint of the contents matches -- an FNV-1a hash over 1024 elements
// sampled at fixed, evenly spread positions plus the first and last column.
// A change to the host buffer that touches none of the sampled elements is
// not detected; callers that modify an operand in place between calls must
// call blasx_serve_invalidate(ptr) (the reference has no cross-call cache at
// all: it rebuilds its per-GPU caches on every call, blas/dgemm.c:106,114).
//
// Latency of a request = submit -> completion detected by the scheduler.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <future>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "executor.h"
#include "host_pipeline.h"
#include "kernels.h"
#include "ozaki.h"
#include "serving.h"
#include "tile_engine.h"

namespace bx {
namespace serve {

namespace {

using Clock = std::chrono::steady_clock;

double now_s() {
    return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Admission: how many pending requests one pass examines, and how long (s)
// the oldest one may be passed by later requests that fit in memory.
constexpr int kLookahead = 64;
constexpr double kHeadWait = 0.05;
// Residue-GEMM tiles per CTA on the emulated path: ~2 ms of one SM at
// K = 16384, after which the SM can take a CTA of another request.
constexpr int kResidueTilesPerCta = 32;

// ---- host-buffer pinning shared by all requests --------------------------------
std::mutex g_pin_mu;
std::map<const void *, std::pair<int, bool>> g_pins;  // ptr -> (users, registered by us)

void pin_acquire(const void *p, size_t bytes) {
    if (!p || !bytes) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pins.find(p);
    if (it != g_pins.end()) {
        it->second.first++;
        return;
    }
    bool ours = false;
    cudaPointerAttributes attr;
    if (!(cudaPointerGetAttributes(&attr, p) == cudaSuccess && attr.type == cudaMemoryTypeHost)) {
        cudaGetLastError();
        ours = cudaHostRegister(const_cast<void *>(p), bytes, cudaHostRegisterDefault) == cudaSuccess;
        if (!ours) cudaGetLastError();
    }
    g_pins[p] = {1, ours};
}

void pin_release(const void *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pins.find(p);
    if (it == g_pins.end()) return;
    if (--it->second.first == 0) {
        if (it->second.second) cudaHostUnregister(const_cast<void *>(p));
        g_pins.erase(it);
    }
}

// ---- operand cache ------------------------------------------------------------------
struct Key {
    const void *ptr;
    int64_t ld, rows, cols;
    int dt;
    uint64_t fp;
    bool operator==(const Key &o) const {
        return ptr == o.ptr && ld == o.ld && rows == o.rows && cols == o.cols && dt == o.dt &&
               fp == o.fp;
    }
};
struct KeyHash {
    size_t operator()(const Key &k) const {
        return std::hash<const void *>()(k.ptr) ^ (size_t(k.fp) * 31u) ^ size_t(k.ld * 131 + k.cols);
    }
};
struct Entry {
    Key key;
    void *dev = nullptr;
    int64_t dld = 0;
    size_t bytes = 0;
    int users = 0;
    bool stale = false;
    std::list<Entry *>::iterator lru;
};

uint64_t fingerprint(const void *p, int64_t ld, int64_t rows, int64_t cols, size_t es) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const unsigned char *b) {
        for (size_t i = 0; i < es; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    };
    const unsigned char *base = static_cast<const unsigned char *>(p);
    const int64_t n = rows * cols;
    if (n == 0) return h;
    auto at = [&](int64_t r, int64_t c) { return base + (r + c * ld) * int64_t(es); };
    for (int t = 0; t < 1024; ++t) {
        const int64_t idx = (int64_t(t) * (n - 1)) / 1023;
        mix(at(idx % rows, idx / rows));
    }
    for (int64_t r = 0; r < rows; ++r) {
        mix(at(r, 0));
        mix(at(r, cols - 1));
    }
    return h;
}

// ---- device memory ---------------------------------------------------------------------
// The serving loop's device memory: one allocation of the HBM budget, made at
// start, cut into 256-byte-aligned blocks first-fit by the scheduler thread
// (the only thread that takes or returns blocks); a returned block merges
// with free neighbours. A request's blocks are returned only after its last
// event has completed, so a block can be reused at once, by any stream.
// Requests never call the stream-ordered allocator, whose pool growth and
// reclaim block the calling thread (they stalled the whole queue).
class Arena {
public:
    int init(size_t bytes) {
        size_ = bytes & ~size_t(255);
        if (size_ == 0) return set_error(BLASX_ERR_ARG, "serving: HBM budget of %zu bytes", bytes);
        if (dev_malloc(reinterpret_cast<void **>(&base_), size_) != cudaSuccess) {
            cudaGetLastError();
            base_ = nullptr;
            return set_error(BLASX_ERR_NOMEM, "serving: cannot reserve the HBM budget of %zu bytes", size_);
        }
        free_[0] = size_;
        return BLASX_OK;
    }
    void release() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
        free_.clear();
        used_.clear();
    }
    size_t size() const { return size_; }
    void *alloc(size_t bytes) {
        bytes = (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > bytes) free_[off + bytes] = len - bytes;
            used_[off] = bytes;
            return base_ + off;
        }
        return nullptr;
    }
    void release_block(void *p) {
        if (!p) return;
        const size_t off = size_t(static_cast<char *>(p) - base_);
        auto u = used_.find(off);
        if (u == used_.end()) return;
        size_t start = off, len = u->second;
        used_.erase(u);
        auto next = free_.lower_bound(start);
        if (next != free_.end() && next->first == start + len) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == start) {
                start = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        free_[start] = len;
    }

private:
    char *base_ = nullptr;
    size_t size_ = 0;
    std::map<size_t, size_t> free_;            // offset -> length
    std::unordered_map<size_t, size_t> used_;  // offset -> length
};

// ---- requests -----------------------------------------------------------------------
struct Request {
    Gemm g;
    double t_submit = 0, t_done = 0;
    double t_admit = 0, t_in = 0, t_exec = 0;  // admitted, copies in landed, executor done
    std::promise<int> done;
    int status = BLASX_OK;
    // device side
    void *dA = nullptr, *dB = nullptr, *dC = nullptr;
    void *ws = nullptr;     // emulated path: its scratch
    bool emulated = false;  // chosen at submission
    int64_t lda = 0, ldb = 0, ldc = 0;
    Entry *bcache = nullptr;  // cached B in use
    Key bkey{};
    bool bkey_valid = false;
    bool on_exec = false;  // computed by the persistent executor
    int stream_slot = -1;
    cudaEvent_t ev_in = nullptr, ev_done = nullptr;
    int stage = 0;  // 1 copying in, 2 on the executor, 3 copying out, 4 failed
    double flops = 0;
    blasx_call_stats stats{};
};

struct Server {
    size_t budget = 0, cache_budget = 0;
    int max_inflight = 8;

    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::shared_ptr<Request>> queue;
    bool stopping = false;
    std::thread thread;

    // scheduler-owned
    std::vector<cudaStream_t> streams;
    std::vector<bool> stream_busy;
    std::vector<std::shared_ptr<Request>> pending, inflight;
    Arena arena;
    exec::Executor *ex = nullptr;
    long long exec_launch_base = 0;  // executor launches before the last statistics reset
    int *err_words = nullptr;  // pinned, one per stream slot: the emulated path's device error word

    std::mutex cache_mu;
    std::unordered_map<Key, Entry *, KeyHash> cache;
    std::list<Entry *> lru;  // front = most recent
    size_t cache_bytes = 0;

    // statistics
    std::mutex stat_mu;
    std::vector<double> latencies;
    double flops = 0, t_first = 0, t_last = 0;
    long long submitted = 0, completed = 0, hits = 0, misses = 0, grouped_launches = 0,
              grouped_requests = 0, failed = 0, memory_waits = 0, head_holds = 0;
    int max_seen = 0;
    double admit_s = 0, admit_max_s = 0;
    double alloc_s = 0, copy_s = 0, enqueue_s = 0;  // parts of admit_s
    double phase_in_s = 0, phase_exec_s = 0, phase_out_s = 0;  // executor requests: summed phases
    long long phase_n = 0;
};

std::mutex g_server_mu;
Server *g_server = nullptr;
std::atomic<bool> g_active{false};

// Drops unused cache entries from the least recently used end while `over`
// holds (caller holds cache_mu; scheduler thread). Returns how many.
template <typename Pred> int evict_lru(Server &s, Pred over) {
    int n = 0;
    auto it = s.lru.end();
    while (it != s.lru.begin() && over()) {
        --it;
        Entry *e = *it;
        if (e->users) continue;
        it = s.lru.erase(it);  // next element: already visited going backwards
        s.cache.erase(e->key);
        s.cache_bytes -= e->bytes;
        s.arena.release_block(e->dev);
        delete e;
        ++n;
    }
    return n;
}

// The emulated scratch for g when its device A and B are separate buffers
// (the loop copies B on its own, or takes it from the operand cache, even
// when the caller passed the same host buffer twice, as SYRK does).
size_t scratch_bytes_separate_b(const Gemm &g) {
    Gemm probe = g;
    probe.B = nullptr;
    return ozaki_scratch_bytes(probe);
}

// Takes a request's device blocks from the arena: A, B (unless a cached copy
// is used), C and the emulated path's scratch, evicting unused cached
// operands (least recently used first) while a block does not fit. Returns
// false, holding nothing, when they still do not fit.
bool reserve(Server &s, Request *r, bool need_b) {
    const Gemm &g = r->g;
    const size_t es = elem_size(g.dt);
    const bool need_ab = !(g.alpha_zero() || g.K == 0);
    r->lda = round_up(g.rows_a(), 32);
    r->ldb = round_up(g.rows_b(), 32);
    r->ldc = round_up(g.M, 32);
    void **dst[4] = {&r->dA, &r->dB, &r->dC, &r->ws};
    const size_t bytes[4] = {need_ab ? size_t(r->lda) * g.cols_a() * es : 0,
                             need_ab && need_b ? size_t(r->ldb) * g.cols_b() * es : 0,
                             size_t(r->ldc) * g.N * es,
                             need_ab && r->emulated ? scratch_bytes_separate_b(g) : 0};
    for (int k = 0; k < 4; ++k) {
        if (!bytes[k]) continue;
        void *p = s.arena.alloc(bytes[k]);
        while (!p) {
            int freed;
            {
                std::lock_guard<std::mutex> lk(s.cache_mu);
                bool once = true;
                freed = evict_lru(s, [&] { const bool o = once; once = false; return o; });
            }
            if (!freed) break;
            p = s.arena.alloc(bytes[k]);
        }
        if (!p) {
            for (int j = 0; j < k; ++j) {
                s.arena.release_block(*dst[j]);
                *dst[j] = nullptr;
            }
            return false;
        }
        *dst[k] = p;
    }
    return true;
}

// Adds the host time of one enqueue call to a scheduler counter.
struct HostTimer {
    double &acc;
    double t0;
    explicit HostTimer(double &a) : acc(a), t0(now_s()) {}
    ~HostTimer() { acc += now_s() - t0; }
};

int admit(Server &s, Request *r, int slot) {
    Gemm &g = r->g;
    const size_t es = elem_size(g.dt);
    cudaStream_t st = s.streams[size_t(slot)];
    r->stream_slot = slot;
    r->t_admit = now_s();
    const bool need_ab = !(g.alpha_zero() || g.K == 0);
    const bool read_c = !g.beta_zero() || g.uplo != 0;  // a triangular output keeps the rest of C
    BX_CUDA(cudaEventCreateWithFlags(&r->ev_in, cudaEventDisableTiming));
    BX_CUDA(cudaEventCreateWithFlags(&r->ev_done, cudaEventDisableTiming));
    if (need_ab) {
        {
            HostTimer t(s.copy_s);
            BX_CUDA(cudaMemcpy2DAsync(r->dA, r->lda * es, g.A, g.lda * es, g.rows_a() * es, g.cols_a(),
                                      cudaMemcpyHostToDevice, st));
        }
        r->stats.h2d_bytes += double(es) * g.rows_a() * g.cols_a();
        if (r->bcache) {
            r->dB = r->bcache->dev;
            r->ldb = r->bcache->dld;
            r->stats.cache_hits += 1;
        } else {
            HostTimer t(s.copy_s);
            BX_CUDA(cudaMemcpy2DAsync(r->dB, r->ldb * es, g.B, g.ldb * es, g.rows_b() * es,
                                      g.cols_b(), cudaMemcpyHostToDevice, st));
            r->stats.h2d_bytes += double(es) * g.rows_b() * g.cols_b();
            r->stats.cache_misses += 1;
        }
    }
    if (read_c) {
        HostTimer t(s.copy_s);
        BX_CUDA(cudaMemcpy2DAsync(r->dC, r->ldc * es, g.C, g.ldc * es, g.M * es, g.N,
                                  cudaMemcpyHostToDevice, st));
        r->stats.h2d_bytes += double(es) * g.M * g.N;
    }
    Gemm d = g;
    d.A = r->dA; d.lda = r->lda;
    d.B = r->dB; d.ldb = r->ldb;
    d.C = r->dC; d.ldc = r->ldc;
    if (r->on_exec) {
        // the executor runs its tiles once the copies (and its descriptor) landed
        BX_TRY(exec::prepare(s.ex, slot, d, r->emulated, config().dgemm_mode.load(), r->ws, st));
        BX_CUDA(cudaEventRecord(r->ev_in, st));
        r->stage = 1;
        return BLASX_OK;
    }
    BX_CUDA(cudaEventRecord(r->ev_in, st));
    d.max_cta_tiles = kResidueTilesPerCta;  // emulated path: let other requests' kernels in
    {
        HostTimer t(s.enqueue_s);
        if (need_ab && r->emulated) {
            // on the request's own scratch; its device error word (the scratch's
            // first word) comes back with the request
            BX_TRY(ozaki_gemm_in(d, st, config().dgemm_mode.load(), r->ws, context()->num_sms));
            BX_CUDA(cudaMemcpyAsync(&s.err_words[slot], r->ws, sizeof(int), cudaMemcpyDeviceToHost, st));
            r->stats.path = 2;
        } else {
            BX_TRY(device_gemm(d, st));
            r->stats.path = call_stats().path;
        }
    }
    r->stats.moduli = 0;
    BX_CUDA(cudaMemcpy2DAsync(g.C, g.ldc * es, r->dC, r->ldc * es, g.M * es, g.N,
                              cudaMemcpyDeviceToHost, st));
    r->stats.d2h_bytes += double(es) * g.M * g.N;
    BX_CUDA(cudaEventRecord(r->ev_done, st));
    r->stage = 3;
    return BLASX_OK;
}

// Moves the executor's requests along: a request whose copies landed has its
// first stage published; one whose device work completed gets its C copied
// back. Returns whether anything moved.
bool exec_progress(Server &s) {
    bool progress = false;
    for (const auto &rp : s.inflight) {
        Request *r = rp.get();
        if (!r->on_exec) continue;
        if (r->stage == 1) {
            const cudaError_t q = cudaEventQuery(r->ev_in);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) {
                cudaGetLastError();
                r->status = BLASX_ERR_CUDA;
                r->stage = 4;  // failed: finished by the completion pass
                progress = true;
                continue;
            }
            r->t_in = now_s();
            if (exec::start(s.ex, r->stream_slot) != BLASX_OK) {
                r->status = last_status();
                r->stage = 4;
            } else {
                r->stage = 2;
            }
            progress = true;
        } else if (r->stage == 2) {
            const int rc = exec::advance(s.ex, r->stream_slot);
            if (rc == 0) continue;
            progress = true;
            r->t_exec = now_s();
            int path = 1, moduli = 0;
            exec::path_of(s.ex, r->stream_slot, &path, &moduli);
            r->stats.path = path;
            r->stats.moduli = moduli;
            if (rc < 0) {
                set_error(BLASX_ERR_TIMEOUT, "serving: a bounded device wait of the executor ran out");
                r->status = BLASX_ERR_TIMEOUT;
                r->stage = 4;
                continue;
            }
            cudaStream_t st = s.streams[size_t(r->stream_slot)];
            const Gemm &g = r->g;
            const size_t es = elem_size(g.dt);
            if (cudaMemcpy2DAsync(g.C, g.ldc * es, r->dC, r->ldc * es, g.M * es, g.N, cudaMemcpyDeviceToHost,
                                  st) != cudaSuccess ||
                cudaEventRecord(r->ev_done, st) != cudaSuccess) {
                cudaGetLastError();
                r->status = BLASX_ERR_CUDA;
                r->stage = 4;
                continue;
            }
            r->stats.d2h_bytes += double(es) * g.M * g.N;
            r->stage = 3;
            std::lock_guard<std::mutex> lk(s.stat_mu);
            s.grouped_requests += 1;
        }
    }
    exec::pump(s.ex);
    return progress;
}

void finish(Server &s, Request *r, int status) {
    cudaStream_t st = s.streams[size_t(r->stream_slot)];
    const Gemm &g = r->g;
    const size_t es = elem_size(g.dt);
    if (status != BLASX_OK) {
        // a request that failed part-way may still have copies in flight on
        // its stream: its blocks go back to the arena only after them
        cudaStreamSynchronize(st);
        cudaGetLastError();
    }
    if (r->emulated && r->ws && status == BLASX_OK && s.err_words[r->stream_slot] != 0) {
        set_error(BLASX_ERR_TIMEOUT, "serving: emulated GEMM's bounded device wait expired (flag %d)",
                  s.err_words[r->stream_slot]);
        status = BLASX_ERR_TIMEOUT;
    }
    s.arena.release_block(r->dA);
    s.arena.release_block(r->dC);
    s.arena.release_block(r->ws);
    {
        std::lock_guard<std::mutex> lk(s.cache_mu);
        if (r->bcache) {
            r->bcache->users--;
            if (r->bcache->stale && r->bcache->users == 0) {
                s.lru.erase(r->bcache->lru);
                s.cache.erase(r->bcache->key);
                s.cache_bytes -= r->bcache->bytes;
                s.arena.release_block(r->bcache->dev);
                delete r->bcache;
            }
        } else if (r->dB) {
            const size_t bytes = size_t(r->ldb) * g.cols_b() * es;
            const bool keep = status == BLASX_OK && r->bkey_valid && bytes <= s.cache_budget &&
                              s.cache.find(r->bkey) == s.cache.end();
            if (keep)  // make room inside the cache budget (least recently used, unused first)
                evict_lru(s, [&] { return s.cache_bytes + bytes > s.cache_budget; });
            if (keep && s.cache_bytes + bytes <= s.cache_budget) {
                Entry *e = new Entry;
                e->key = r->bkey;
                e->dev = r->dB;
                e->dld = r->ldb;
                e->bytes = bytes;
                s.lru.push_front(e);
                e->lru = s.lru.begin();
                s.cache[e->key] = e;
                s.cache_bytes += bytes;
            } else {
                s.arena.release_block(r->dB);
            }
        }
    }
    s.stream_busy[size_t(r->stream_slot)] = false;
    if (r->ev_in) cudaEventDestroy(r->ev_in);
    if (r->ev_done) cudaEventDestroy(r->ev_done);
    r->t_done = now_s();
    r->stats.seconds = r->t_done - r->t_submit;
    {
        std::lock_guard<std::mutex> lk(s.stat_mu);
        if (r->on_exec && status == BLASX_OK && r->t_exec > 0) {
            s.phase_in_s += r->t_in - r->t_admit;
            s.phase_exec_s += r->t_exec - r->t_in;
            s.phase_out_s += r->t_done - r->t_exec;
            s.phase_n += 1;
        }
        s.completed += 1;
        if (status != BLASX_OK) s.failed += 1;
        s.latencies.push_back(r->t_done - r->t_submit);
        s.flops += g.flops();
        s.t_last = r->t_done;
    }
    r->status = status;
    r->done.set_value(status);
}

// A request larger than the whole budget: the library's own host path (in
// core, or out of core through the tile cache, with its own device memory)
// runs it on the scheduler thread while nothing else is in flight.
void run_alone(Server &s, Request *r) {
    const int st = host_gemm(r->g);
    r->stats = call_stats();
    r->t_done = now_s();
    {
        std::lock_guard<std::mutex> lk(s.stat_mu);
        s.completed += 1;
        if (st != BLASX_OK) s.failed += 1;
        s.latencies.push_back(r->t_done - r->t_submit);
        s.flops += r->g.flops();
        s.t_last = r->t_done;
    }
    r->status = st;
    r->done.set_value(st);
}

void loop(Server *sp) {
    Server &s = *sp;
    Context *c = context();
    if (c) cudaSetDevice(c->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s.mu);
            if (s.pending.empty() && s.inflight.empty()) {
                if (s.queue.empty() && !s.stopping) {
                    // nothing to do: give the SMs back before sleeping
                    lk.unlock();
                    exec::stop(s.ex);
                    lk.lock();
                }
                s.cv.wait(lk, [&] { return s.stopping || !s.queue.empty(); });
                if (s.stopping && s.queue.empty()) return;
            }
            while (!s.queue.empty()) {
                s.pending.push_back(s.queue.front());
                s.queue.pop_front();
            }
        }
        bool progress = false;
        // completions
        for (size_t i = 0; i < s.inflight.size();) {
            Request *r = s.inflight[i].get();
            if (r->stage == 4) {
                finish(s, r, r->status != BLASX_OK ? r->status : BLASX_ERR_CUDA);
                s.inflight.erase(s.inflight.begin() + long(i));
                progress = true;
                continue;
            }
            if (r->stage == 3) {
                const cudaError_t q = cudaEventQuery(r->ev_done);
                if (q == cudaSuccess || (q != cudaErrorNotReady)) {
                    if (q != cudaSuccess) cudaGetLastError();
                    finish(s, r, q == cudaSuccess ? BLASX_OK : BLASX_ERR_CUDA);
                    s.inflight.erase(s.inflight.begin() + long(i));
                    progress = true;
                    continue;
                }
            }
            ++i;
        }
        // the executor's requests: publish stages, copy finished results back
        if (exec_progress(s)) progress = true;
        // admission: arrival order, except that while the oldest pending
        // request waits for memory, up to kLookahead requests behind it that
        // fit may pass it -- until it has waited kHeadWait; from then on
        // nothing passes it, so the memory that finishing requests free
        // goes to it
        size_t idx = 0;
        int scanned = 0;
        const double now = now_s();
        while (idx < s.pending.size() && int(s.inflight.size()) < s.max_inflight &&
               scanned < kLookahead) {
            std::shared_ptr<Request> rp = s.pending[idx];
            Request *r = rp.get();
            ++scanned;
            if (!r->on_exec) {
                // SYMM / HEMM operand forms and Hermitian outputs run on their own
                // kernels, which cannot share the SMs with the executor: only
                // when nothing else is in flight, with the executor stopped
                if (!s.inflight.empty()) {
                    if (idx == 0) break;  // keeps its place at the head
                    ++idx;
                    continue;
                }
                exec::stop(s.ex);
            }
            // operand cache lookup for B
            Entry *hit = nullptr;
            {
                std::lock_guard<std::mutex> lk(s.cache_mu);
                if (r->bkey_valid) {
                    auto it = s.cache.find(r->bkey);
                    if (it != s.cache.end() && !it->second->stale) {
                        hit = it->second;
                        hit->users++;
                        s.lru.splice(s.lru.begin(), s.lru, hit->lru);
                    }
                }
            }
            int slot = -1;
            for (size_t k = 0; k < s.stream_busy.size(); ++k)
                if (!s.stream_busy[k]) { slot = int(k); break; }
            if (slot < 0) {
                if (hit) {
                    std::lock_guard<std::mutex> lk(s.cache_mu);
                    hit->users--;
                }
                break;
            }
            bool fits;
            {
                HostTimer t(s.alloc_s);
                fits = reserve(s, r, hit == nullptr);
            }
            if (!fits) {
                if (hit) {
                    std::lock_guard<std::mutex> lk(s.cache_mu);
                    hit->users--;
                }
                if (s.inflight.empty()) {  // larger than the whole budget
                    s.pending.erase(s.pending.begin() + long(idx));
                    run_alone(s, r);
                    progress = true;
                    continue;
                }
                {
                    std::lock_guard<std::mutex> lk(s.stat_mu);
                    ++s.memory_waits;
                    if (idx == 0 && now - r->t_submit > kHeadWait) ++s.head_holds;
                }
                if (idx == 0 && now - r->t_submit > kHeadWait) break;  // memory is kept for it
                ++idx;  // does not fit yet: look further back
                continue;
            }
            s.pending.erase(s.pending.begin() + long(idx));
            s.stream_busy[size_t(slot)] = true;
            r->bcache = hit;
            {
                std::lock_guard<std::mutex> lk(s.stat_mu);
                if (r->bkey_valid && !(r->g.alpha_zero() || r->g.K == 0)) (hit ? s.hits : s.misses) += 1;
            }
            const double a0 = now_s();
            const int st = admit(s, r, slot);
            {
                const double da = now_s() - a0;
                std::lock_guard<std::mutex> lk(s.stat_mu);
                s.admit_s += da;
                s.admit_max_s = std::max(s.admit_max_s, da);
            }
            s.inflight.push_back(rp);
            s.max_seen = std::max(s.max_seen, int(s.inflight.size()));
            if (st != BLASX_OK) {
                s.inflight.pop_back();
                finish(s, r, st);
            }
            progress = true;
        }
        // requests on the executor move on its completions: poll them closely
        if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(s.inflight.empty() ? 50 : 10));
    }
}

}  // namespace

bool active() { return g_active.load(std::memory_order_acquire); }

int submit(const Gemm &g) {
    Server *s;
    {
        std::lock_guard<std::mutex> lk(g_server_mu);
        s = g_server;
    }
    if (!s) return set_error(BLASX_ERR_CLOSED, "serving loop is not running");
    const size_t es = elem_size(g.dt);
    const bool need_ab = !(g.alpha_zero() || g.K == 0);
    // shared by the caller and the scheduler: whichever lets go last frees it
    auto rp = std::make_shared<Request>();
    Request *r = rp.get();
    r->g = g;
    r->t_submit = now_s();
    r->flops = 0;
    r->emulated = need_ab && ozaki_selected(g, config().dgemm_mode.load());
    r->on_exec = exec::supports(g);
    if (need_ab) {
        r->bkey = Key{g.B, g.ldb, g.rows_b(), g.cols_b(), int(g.dt),
                      fingerprint(g.B, g.ldb, g.rows_b(), g.cols_b(), es)};
        r->bkey_valid = true;
    }
    pin_acquire(g.A, need_ab ? host_extent(g.lda, g.rows_a(), g.cols_a(), es) : 0);
    pin_acquire(g.B, need_ab ? host_extent(g.ldb, g.rows_b(), g.cols_b(), es) : 0);
    pin_acquire(g.C, host_extent(g.ldc, g.M, g.N, es));
    std::future<int> fut = r->done.get_future();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return set_error(BLASX_ERR_CLOSED, "serving loop is shutting down");
        s->queue.push_back(rp);
        std::lock_guard<std::mutex> lk2(s->stat_mu);
        s->submitted += 1;
        if (s->t_first == 0) s->t_first = r->t_submit;
    }
    s->cv.notify_one();
    const int st = fut.get();
    pin_release(g.A);
    pin_release(g.B);
    pin_release(g.C);
    call_stats() = r->stats;
    if (call_stats().path == 0) call_stats().path = 1;
    if (st != BLASX_OK) return set_error(st, "serving: request failed");
    return BLASX_OK;
}

}  // namespace serve
}  // namespace bx

using namespace bx::serve;

extern "C" {

int blasx_serve_start(size_t hbm_budget, size_t cache_bytes, int max_inflight) {
    std::lock_guard<std::mutex> lk(g_server_mu);
    if (g_server) return BLASX_OK;
    bx::Context *c = bx::context();
    if (!c) return bx::last_status();
    auto *s = new Server;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = hbm_budget ? hbm_budget : size_t(double(free_b) * 0.85);
    s->cache_budget = cache_bytes ? std::min(cache_bytes, s->budget / 2) : s->budget / 4;
    s->max_inflight = max_inflight > 0 ? std::min(max_inflight, 64) : 8;
    int rc = s->arena.init(s->budget);
    if (rc == BLASX_OK) rc = bx::oz::upload_crt_tables();
    if (rc == BLASX_OK) rc = bx::exec::create(s->max_inflight, &s->ex);
    if (rc == BLASX_OK && cudaHostAlloc(reinterpret_cast<void **>(&s->err_words),
                                        sizeof(int) * size_t(s->max_inflight), cudaHostAllocDefault) != cudaSuccess)
        rc = bx::set_error(BLASX_ERR_NOMEM, "serving: pinned error words");
    if (rc != BLASX_OK) {
        bx::exec::destroy(s->ex);
        s->arena.release();
        delete s;
        return rc;
    }
    memset(s->err_words, 0, sizeof(int) * size_t(s->max_inflight));
    s->streams.resize(size_t(s->max_inflight));
    s->stream_busy.assign(size_t(s->max_inflight), false);
    // the requests' streams carry their copies (and, for requests the executor
    // does not run, their kernels)
    for (auto &st : s->streams) cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    s->thread = std::thread(loop, s);
    g_server = s;
    g_active.store(true, std::memory_order_release);
    return BLASX_OK;
}

int blasx_serve_stop(void) {
    Server *s;
    {
        std::lock_guard<std::mutex> lk(g_server_mu);
        s = g_server;
        if (!s) return BLASX_OK;
        g_active.store(false, std::memory_order_release);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv.notify_all();
    s->thread.join();  // the loop drains queued and in-flight requests first
    bx::exec::destroy(s->ex);
    {
        std::lock_guard<std::mutex> lk(s->cache_mu);
        for (auto &kv : s->cache) delete kv.second;
    }
    for (auto st : s->streams) cudaStreamDestroy(st);
    s->arena.release();
    cudaFreeHost(s->err_words);
    std::lock_guard<std::mutex> lk(g_server_mu);
    g_server = nullptr;
    delete s;
    return BLASX_OK;
}

int blasx_serve_invalidate(const void *host_ptr) {
    std::lock_guard<std::mutex> lk(g_server_mu);
    if (!g_server) return BLASX_OK;
    Server &s = *g_server;
    std::lock_guard<std::mutex> lk2(s.cache_mu);
    int n = 0;
    for (auto &kv : s.cache)
        if (kv.first.ptr == host_ptr) {
            kv.second->stale = true;
            ++n;
        }
    return n;
}

void blasx_serve_get_stats(blasx_serve_stats *out) {
    if (!out) return;
    memset(out, 0, sizeof *out);
    std::lock_guard<std::mutex> lk(g_server_mu);
    if (!g_server) return;
    Server &s = *g_server;
    std::lock_guard<std::mutex> lk2(s.stat_mu);
    out->submitted = s.submitted;
    out->completed = s.completed;
    out->failed = s.failed;
    out->cache_hits = s.hits;
    out->cache_misses = s.misses;
    {
        long long launches = 0, tasks = 0;
        bx::exec::counters(s.ex, &launches, &tasks);
        out->grouped_launches = launches - s.exec_launch_base;
    }
    out->grouped_requests = s.grouped_requests;
    out->max_inflight_seen = s.max_seen;
    out->flops = s.flops;
    out->seconds = s.t_last > s.t_first ? s.t_last - s.t_first : 0;
    out->tflops = out->seconds > 0 ? s.flops / out->seconds / 1e12 : 0;
    out->admit_seconds = s.admit_s;
    out->admit_max_ms = s.admit_max_s * 1e3;
    out->memory_waits = s.memory_waits;
    out->head_holds = s.head_holds;
    out->alloc_seconds = s.alloc_s;
    out->copy_seconds = s.copy_s;
    out->compute_enqueue_seconds = s.enqueue_s;
    if (s.phase_n) {
        out->mean_copy_in_ms = s.phase_in_s / double(s.phase_n) * 1e3;
        out->mean_compute_ms = s.phase_exec_s / double(s.phase_n) * 1e3;
        out->mean_copy_out_ms = s.phase_out_s / double(s.phase_n) * 1e3;
    }
    if (!s.latencies.empty()) {
        std::vector<double> l = s.latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const size_t i = std::min(l.size() - 1, size_t(q * double(l.size() - 1) + 0.5));
            return l[i] * 1e3;
        };
        double sum = 0;
        for (double v : l) sum += v;
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->mean_ms = sum / double(l.size()) * 1e3;
        out->max_ms = l.back() * 1e3;
    }
}

int blasx_serve_reset_stats(void) {
    std::lock_guard<std::mutex> lk(g_server_mu);
    if (!g_server) return BLASX_OK;
    Server &s = *g_server;
    std::lock_guard<std::mutex> lk2(s.stat_mu);
    s.latencies.clear();
    s.flops = 0;
    s.t_first = s.t_last = 0;
    s.submitted = s.completed = s.hits = s.misses = s.grouped_launches = s.grouped_requests = 0;
    {
        long long launches = 0, tasks = 0;
        bx::exec::counters(s.ex, &launches, &tasks);
        s.exec_launch_base = launches;
    }
    s.failed = 0;
    s.max_seen = 0;
    s.memory_waits = s.head_holds = 0;
    s.admit_s = s.admit_max_s = 0;
    s.alloc_s = s.copy_s = s.enqueue_s = 0;
    s.phase_in_s = s.phase_exec_s = s.phase_out_s = 0;
    s.phase_n = 0;
    return BLASX_OK;
}

}  // extern "C"
