// staging.cu -- pinned bounce buffers for the pageable host memory of host
// GEMM calls (the design is described in staging.h).
#include "staging.h"

#include <algorithm>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>

namespace bx {
namespace {

constexpr size_t kPiece = size_t(32) << 20;  // bytes of one bounce buffer
constexpr int kRing = 8;                      // buffers per direction

thread_local HostPin *t_top = nullptr;  // the thread's innermost call with staged ranges

// Threads that split one copy among themselves; the submitting thread takes
// part, so a job completes even when every worker is busy elsewhere.
class Workers {
public:
    explicit Workers(int n) {
        for (int i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
    }
    int size() const { return int(th_.size()) + 1; }
    // Runs fn(0) .. fn(parts - 1); returns when all of them have returned.
    void run(int parts, const std::function<void(int)> &fn) {
        if (parts <= 1 || th_.empty()) {
            for (int i = 0; i < parts; ++i) fn(i);
            return;
        }
        Job j;
        j.fn = &fn;
        j.parts = parts;
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(&j);
        }
        cv_.notify_all();
        for (;;) {
            int i;
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (j.next >= parts) break;
                i = j.next++;
                if (j.next == parts) q_.erase(std::find(q_.begin(), q_.end(), &j));
            }
            fn(i);
            std::lock_guard<std::mutex> lk(mu_);
            ++j.done;
        }
        std::unique_lock<std::mutex> lk(mu_);
        j.fin.wait(lk, [&] { return j.done == parts; });
    }

private:
    struct Job {
        const std::function<void(int)> *fn = nullptr;
        int parts = 0, next = 0, done = 0;
        std::condition_variable fin;
    };
    void loop() {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return !q_.empty(); });
            Job *j = q_.front();
            const int i = j->next++;
            if (j->next == j->parts) q_.pop_front();
            lk.unlock();
            (*j->fn)(i);
            lk.lock();
            // notified under the lock: the submitter cannot return (and free
            // the job) before this thread has let go of it
            if (++j->done == j->parts) j->fin.notify_all();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Job *> q_;
    std::vector<std::thread> th_;
};

// Byte range [lo, hi) of a 2-D host region.
struct Span {
    const char *lo, *hi;
    bool overlaps(const Span &o) const { return lo < o.hi && o.lo < hi; }
};
Span span_of(const void *p, size_t pitch, size_t width, size_t height) {
    const char *c = static_cast<const char *>(p);
    return {c, c + (height - 1) * pitch + width};
}

struct Buf {
    char *p = nullptr;
    cudaEvent_t ev = nullptr;  // recorded after the buffer's DMA
    bool used = false;         // ev has been recorded
};

struct CopyOut {
    int buf;
    char *dst;
    size_t dpitch, width, rows;
    HostPin *call;
    long long seq;
};

class Stager {
public:
    Stager() {
        int n = 0;
        if (const char *e = getenv("BLASX_STAGING_THREADS")) n = atoi(e);
        if (n <= 0) n = std::clamp(int(std::thread::hardware_concurrency()) / 2, 1, 16);
        workers_ = new Workers(n - 1);
        writer_ = std::thread([this] { write_loop(); });
        writer_.detach();
    }

    int h2d(char *dst, size_t dpitch, const char *src, size_t spitch, size_t width, size_t height,
            cudaStream_t s) {
        std::lock_guard<std::mutex> sub(submit_mu_);
        BX_TRY(ensure());
        BX_TRY(wait_overlapping(span_of(src, spitch, width, height)));
        return pieces(width, height, [&](size_t r0, size_t off, size_t w, size_t rows) -> int {
            Buf &b = in_[in_next_];
            in_next_ = (in_next_ + 1) % kRing;
            if (b.used) BX_CUDA(cudaEventSynchronize(b.ev));  // its previous DMA has read it
            copy_rows(b.p, w, src + r0 * spitch + off, spitch, w, rows);
            BX_CUDA(cudaMemcpy2DAsync(dst + r0 * dpitch + off, dpitch, b.p, w, w, rows,
                                      cudaMemcpyHostToDevice, s));
            BX_CUDA(cudaEventRecord(b.ev, s));
            b.used = true;
            return BLASX_OK;
        });
    }

    int d2h(char *dst, size_t dpitch, const char *src, size_t spitch, size_t width, size_t height,
            cudaStream_t s, HostPin *call) {
        std::lock_guard<std::mutex> sub(submit_mu_);
        BX_TRY(ensure());
        return pieces(width, height, [&](size_t r0, size_t off, size_t w, size_t rows) -> int {
            int idx;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return !out_busy_[out_next_]; });  // its copy-out has finished
                idx = out_next_;
                out_next_ = (out_next_ + 1) % kRing;
                out_busy_[idx] = true;
            }
            Buf &b = out_[idx];
            cudaError_t e = cudaMemcpy2DAsync(b.p, w, src + r0 * spitch + off, spitch, w, rows,
                                              cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaEventRecord(b.ev, s);
            std::lock_guard<std::mutex> lk(mu_);
            if (e != cudaSuccess) {
                out_busy_[idx] = false;
                return set_error(BLASX_ERR_CUDA, "staged device-to-host copy: %s", cudaGetErrorString(e));
            }
            call->pending.fetch_add(1);
            q_.push_back(CopyOut{idx, dst + r0 * dpitch + off, dpitch, w, rows, call, ++submitted_});
            cv_.notify_all();
            return BLASX_OK;
        });
    }

    // Waits until no copy-out of `call` is pending.
    int wait_call(HostPin *call) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return call->pending.load() == 0; });
        return call->error.load();
    }

    void release() {
        std::lock_guard<std::mutex> sub(submit_mu_);
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return q_.empty(); });
        }
        for (Buf *ring : {in_, out_})
            for (int i = 0; i < kRing; ++i) {
                if (ring[i].ev) cudaEventDestroy(ring[i].ev);
                if (ring[i].p) cudaFreeHost(ring[i].p);
                ring[i] = Buf{};
            }
        ready_ = false;
    }

private:
    int ensure() {
        if (ready_) return BLASX_OK;
        cudaGetDevice(&device_);
        for (Buf *ring : {in_, out_})
            for (int i = 0; i < kRing; ++i) {
                if (!ring[i].p) BX_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&ring[i].p), kPiece,
                                                      cudaHostAllocPortable));
                if (!ring[i].ev)
                    BX_CUDA(cudaEventCreateWithFlags(&ring[i].ev, cudaEventDisableTiming | cudaEventBlockingSync));
                ring[i].used = false;
            }
        in_next_ = out_next_ = 0;
        ready_ = true;
        return BLASX_OK;
    }

    // Cuts a region of height rows of width bytes into pieces of at most one
    // buffer: whole rows, or (a row longer than a buffer) one row's segments.
    template <class F>
    int pieces(size_t width, size_t height, F &&fn) {
        if (width <= kPiece) {
            const size_t per = kPiece / width;
            for (size_t r0 = 0; r0 < height; r0 += per) BX_TRY(fn(r0, 0, width, std::min(per, height - r0)));
        } else {
            for (size_t r = 0; r < height; ++r)
                for (size_t off = 0; off < width; off += kPiece) BX_TRY(fn(r, off, std::min(kPiece, width - off), 1));
        }
        return BLASX_OK;
    }

    // rows of width bytes between pitched regions, split among the workers
    // by rows (or, with fewer rows than workers, by byte ranges of each row)
    void copy_rows(char *dst, size_t dpitch, const char *src, size_t spitch, size_t width, size_t rows) {
        const int parts = width * rows < (size_t(1) << 20) ? 1 : workers_->size();
        const bool by_rows = rows >= size_t(parts);
        workers_->run(parts, [&](int i) {
            if (by_rows) {
                const size_t a = rows * i / parts, b = rows * (i + 1) / parts;
                for (size_t r = a; r < b; ++r) memcpy(dst + r * dpitch, src + r * spitch, width);
            } else {
                const size_t a = width * i / parts, b = width * (i + 1) / parts;
                for (size_t r = 0; r < rows; ++r) memcpy(dst + r * dpitch + a, src + r * spitch + a, b - a);
            }
        });
    }

    // A staged read of host memory that a pending copy-out will write waits
    // for that copy-out (copy-outs finish in submission order).
    int wait_overlapping(const Span &sp) {
        std::unique_lock<std::mutex> lk(mu_);
        long long last = 0;
        for (const CopyOut &j : q_)
            if (sp.overlaps(span_of(j.dst, j.dpitch, j.width, j.rows))) last = j.seq;
        if (last) cv_.wait(lk, [&] { return finished_ >= last; });
        return BLASX_OK;
    }

    void write_loop() {
        std::unique_lock<std::mutex> lk(mu_);
        bool device_set = false;
        for (;;) {
            cv_.wait(lk, [&] { return !q_.empty(); });
            const CopyOut j = q_.front();  // stays queued (for overlap checks) until written
            lk.unlock();
            if (!device_set) {
                cudaSetDevice(device_);
                device_set = true;
            }
            const cudaError_t e = cudaEventSynchronize(out_[j.buf].ev);
            if (e == cudaSuccess) copy_rows(j.dst, j.dpitch, out_[j.buf].p, j.width, j.width, j.rows);
            lk.lock();
            if (e != cudaSuccess) j.call->error.store(BLASX_ERR_CUDA);
            q_.pop_front();
            out_busy_[j.buf] = false;
            finished_ = j.seq;
            j.call->pending.fetch_sub(1);  // the call may end once this is 0: not touched after
            cv_.notify_all();
        }
    }

    std::mutex submit_mu_;  // one submitting thread at a time (the rings' order)
    std::mutex mu_;         // the outbound ring and the copy-out queue
    std::condition_variable cv_;
    Buf in_[kRing], out_[kRing];
    bool out_busy_[kRing] = {};
    int in_next_ = 0, out_next_ = 0;
    bool ready_ = false;
    int device_ = 0;
    std::deque<CopyOut> q_;
    long long submitted_ = 0, finished_ = 0;
    Workers *workers_ = nullptr;
    std::thread writer_;
};

// Created on first use and never destroyed: its threads outlive static
// destruction at exit.
Stager &stager() {
    static Stager *s = new Stager;
    return *s;
}
std::atomic<bool> g_stager_made{false};

bool staging_enabled() { return config().host_staging.load() != 0; }

// The innermost call of this thread that staged a range holding p.
HostPin *owner_of(const void *p) {
    const char *c = static_cast<const char *>(p);
    for (HostPin *h = t_top; h; h = h->outer)
        for (const auto &r : h->staged)
            if (c >= r.first && c < r.first + r.second) return h;
    return nullptr;
}

}  // namespace

int HostPin::pin(const void *p, size_t bytes) {
    if (!p || !bytes) return BLASX_OK;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) == cudaSuccess && attr.type != cudaMemoryTypeUnregistered)
        return BLASX_OK;  // pinned or device memory: copied directly
    cudaGetLastError();
    if (staging_enabled()) {
        staged.emplace_back(static_cast<const char *>(p), bytes);
        if (!linked) {
            outer = t_top;
            t_top = this;
            linked = true;
        }
        g_stager_made.store(true);
        return BLASX_OK;
    }
    if (cudaHostRegister(const_cast<void *>(p), bytes, cudaHostRegisterDefault) == cudaSuccess) {
        regs.push_back(const_cast<void *>(p));
    } else {
        cudaGetLastError();  // not registrable: the copies run synchronously through the driver
    }
    return BLASX_OK;
}

int HostPin::finish() {
    if (!linked) return BLASX_OK;
    const int rc = stager().wait_call(this);
    if (rc != BLASX_OK) return set_error(rc, "staged device-to-host copy failed");
    return BLASX_OK;
}

HostPin::~HostPin() {
    if (linked) {
        stager().wait_call(this);
        // calls end in reverse order of their start on one thread
        t_top = outer;
    }
    for (void *p : regs) cudaHostUnregister(p);
}

int copy2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t height,
           cudaMemcpyKind kind, cudaStream_t s) {
    if (width == 0 || height == 0) return BLASX_OK;
    HostPin *call = nullptr;
    if (t_top) {
        if (kind == cudaMemcpyHostToDevice) call = owner_of(src);
        else if (kind == cudaMemcpyDeviceToHost) call = owner_of(dst);
    }
    if (!call) {
        BX_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, kind, s));
        return BLASX_OK;
    }
    if (kind == cudaMemcpyHostToDevice)
        return stager().h2d(static_cast<char *>(dst), dpitch, static_cast<const char *>(src), spitch, width,
                            height, s);
    return stager().d2h(static_cast<char *>(dst), dpitch, static_cast<const char *>(src), spitch, width, height,
                        s, call);
}

void release_staging() {
    if (g_stager_made.load()) stager().release();
}

}  // namespace bx
