// profile.cu -- per-phase CUDA-event timing (see profile.h).
#include <atomic>
#include <mutex>
#include <vector>

#include "profile.h"

namespace bx {
namespace prof {

namespace {
std::atomic<bool> g_on{false};
std::mutex g_mu;
std::vector<cudaEvent_t> g_free;
struct Span {
    int phase;
    cudaEvent_t a, b;
};
std::vector<Span> g_pending;
double g_ms[kNumPhases] = {0, 0, 0, 0};
long g_count[kNumPhases] = {0, 0, 0, 0};

cudaEvent_t take() {
    if (!g_free.empty()) {
        cudaEvent_t e = g_free.back();
        g_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Folds completed spans into the totals (caller holds g_mu). Blocks on
// events that have not completed yet.
void drain() {
    for (const Span &s : g_pending) {
        float ms = 0;
        if (cudaEventSynchronize(s.b) == cudaSuccess && cudaEventElapsedTime(&ms, s.a, s.b) == cudaSuccess) {
            g_ms[s.phase] += ms;
            g_count[s.phase] += 1;
        }
        g_free.push_back(s.a);
        g_free.push_back(s.b);
    }
    g_pending.clear();
}
}  // namespace

bool enabled() { return g_on.load(std::memory_order_relaxed); }

cudaEvent_t mark(cudaStream_t s) {
    if (!enabled()) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEvent_t e = take();
    if (e) cudaEventRecord(e, s);
    return e;
}

void span(int phase, cudaEvent_t a, cudaEvent_t b) {
    if (!a || !b) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_pending.push_back({phase, a, b});
}

}  // namespace prof
}  // namespace bx

extern "C" {

int blasx_profile_enable(int on) {
    std::lock_guard<std::mutex> lk(bx::prof::g_mu);
    bx::prof::drain();
    for (int i = 0; i < bx::prof::kNumPhases; ++i) {
        bx::prof::g_ms[i] = 0;
        bx::prof::g_count[i] = 0;
    }
    return bx::prof::g_on.exchange(on != 0) ? 1 : 0;
}

int blasx_profile_read(double *ms, long *count, int n) {
    std::lock_guard<std::mutex> lk(bx::prof::g_mu);
    bx::prof::drain();
    for (int i = 0; i < n && i < bx::prof::kNumPhases; ++i) {
        if (ms) ms[i] = bx::prof::g_ms[i];
        if (count) count[i] = bx::prof::g_count[i];
    }
    return bx::prof::kNumPhases;
}

}  // extern "C"
