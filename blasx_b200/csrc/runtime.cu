// runtime.cu -- status recording, configuration and the device context.
//
// Replaces the reference's lazily initialised global resources
// (blasx_tile_init / blasx_resource_init, blas/blasx_internal.c:51-90, guarded
// by the global mutex of blas/blasx_mutex.c): one context per process for the
// single B200, created on first use, with dedicated compute / H2D / D2H
// streams. Unlike the reference, failures are reported as a status instead of
// assert()-aborting the host process.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ozaki.h"
#include "runtime.h"
#include "staging.h"
#include "tile_engine.h"

namespace bx {

namespace {
thread_local int t_status = BLASX_OK;
thread_local char t_msg[512] = "";
thread_local blasx_call_stats t_stats{};

std::atomic<uint64_t> g_launches{0};
std::mutex g_ctx_mu;
Context *g_ctx = nullptr;

size_t parse_bytes(const char *s) {
    char *end = nullptr;
    double v = strtod(s, &end);
    if (end && *end) {
        switch (*end) {
            case 'k': case 'K': v *= 1024.0; break;
            case 'm': case 'M': v *= 1024.0 * 1024.0; break;
            case 'g': case 'G': v *= 1024.0 * 1024.0 * 1024.0; break;
            default: break;
        }
    }
    return v > 0 ? size_t(v) : 0;
}

void read_env(Config &c) {
    if (const char *m = getenv("BLASX_DGEMM_MODE")) {
        if (!strcmp(m, "native")) c.dgemm_mode = 1;
        else if (!strcmp(m, "ozaki")) c.dgemm_mode = 2;
        else c.dgemm_mode = 0;
    }
    if (const char *b = getenv("BLASX_HBM_BUDGET")) c.hbm_budget = parse_bytes(b);
    if (const char *t = getenv("BLASX_TILE")) c.tile = atoi(t);
    if (const char *h = getenv("BLASX_HOST_STAGING")) c.host_staging = strcmp(h, "0") && strcmp(h, "off") ? 1 : 0;
}
}  // namespace

int set_error(int status, const char *fmt, ...) {
    t_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof t_msg, fmt, ap);
    va_end(ap);
    if (status != BLASX_OK && status != BLASX_ERR_ARG) fprintf(stderr, "blasx_b200: %s\n", t_msg);
    return status;
}

void clear_error() {
    t_status = BLASX_OK;
    t_msg[0] = 0;
}

int last_status() { return t_status; }

Config &config() {
    static Config c;
    static std::once_flag once;
    std::call_once(once, [] { read_env(c); });
    return c;
}

blasx_call_stats &call_stats() { return t_stats; }

void count_launch(int n) { g_launches.fetch_add(uint64_t(n), std::memory_order_relaxed); }

namespace {
std::atomic<int> g_fail_alloc_countdown{0};  // > 0: the allocation that brings it to 0 fails

bool injected_alloc_failure() {
    int n = g_fail_alloc_countdown.load();
    while (n > 0) {
        if (g_fail_alloc_countdown.compare_exchange_weak(n, n - 1)) return n == 1;
    }
    return false;
}
}  // namespace

cudaError_t dev_malloc_async(void **p, size_t bytes, cudaStream_t s) {
    if (injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocAsync(p, bytes, s);
}

cudaError_t dev_malloc(void **p, size_t bytes) {
    if (injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

void resolve_decision(blasx_call_stats &st) {
    // moduli >= 0: already known (a served request reports its own decision)
    if (st.path != 2 || st.moduli >= 0 || !g_ctx) return;
    const oz::Decision *d = static_cast<const oz::Decision *>(g_ctx->last_decision);
    st.moduli = d->nmod;
    if (d->nmod == 0) st.path = 4;  // native fallback chosen on the device
}

Context *context() {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (g_ctx) {
        cudaSetDevice(g_ctx->device);
        return g_ctx;
    }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error(BLASX_ERR_NODEVICE, "no CUDA device available (%s)",
                  e == cudaSuccess ? "count is 0" : cudaGetErrorString(e));
        return nullptr;
    }
    auto *c = new Context;
    const char *d = getenv("BLASX_DEVICE");
    c->device = d ? atoi(d) : 0;
    if (c->device < 0 || c->device >= n) c->device = 0;
    cudaDeviceProp prop;
    if ((e = cudaSetDevice(c->device)) != cudaSuccess ||
        (e = cudaGetDeviceProperties(&prop, c->device)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->compute, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking)) != cudaSuccess) {
        set_error(BLASX_ERR_CUDA, "device context init failed: %s", cudaGetErrorString(e));
        delete c;
        return nullptr;
    }
    if (prop.major != 10) {
        set_error(BLASX_ERR_NODEVICE,
                  "device %d is sm_%d%d; this library is built for sm_100a (B200) only",
                  c->device, prop.major, prop.minor);
        delete c;
        return nullptr;
    }
    c->num_sms = prop.multiProcessorCount;
    c->total_mem = prop.totalGlobalMem;
    void *pinned = nullptr;
    if ((e = cudaHostAlloc(&pinned, 256, cudaHostAllocDefault)) != cudaSuccess) {
        set_error(BLASX_ERR_CUDA, "pinned slot allocation failed: %s", cudaGetErrorString(e));
        delete c;
        return nullptr;
    }
    memset(pinned, 0, 256);
    c->last_decision = pinned;
    c->last_error_flag = reinterpret_cast<int *>(static_cast<char *>(pinned) + 128);
    // keep freed pool memory cached in the device pool between calls
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, c->device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    g_ctx = c;
    return c;
}

int release_context() {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (!g_ctx) return BLASX_OK;
    cudaSetDevice(g_ctx->device);
    cudaDeviceSynchronize();
    release_tile_arena();
    release_staging();
    cudaStreamDestroy(g_ctx->compute);
    cudaStreamDestroy(g_ctx->h2d);
    cudaStreamDestroy(g_ctx->d2h);
    cudaFreeHost(g_ctx->last_decision);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, g_ctx->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    delete g_ctx;
    g_ctx = nullptr;
    return BLASX_OK;
}

}  // namespace bx

extern "C" {

int blasx_last_status(void) { return bx::last_status(); }

const char *blasx_last_error(void) { return bx::t_msg; }

int blasx_set_dgemm_mode(int mode) {
    if (mode < 0 || mode > 2) return -1;
    return bx::config().dgemm_mode.exchange(mode);
}

int blasx_set_hbm_budget(size_t bytes) {
    bx::config().hbm_budget = bytes;
    return 0;
}

int blasx_set_host_staging(int on) { return bx::config().host_staging.exchange(on ? 1 : 0); }

int blasx_set_tile(int tile) {
    if (tile != 0 && (tile < 256 || tile > 16384 || tile % 256)) return -1;
    bx::config().tile = tile;
    return 0;
}

void blasx_get_call_stats(blasx_call_stats *out) {
    if (!out) return;
    *out = bx::call_stats();
    bx::resolve_decision(*out);
}

int blasx_finalize(void) { return bx::release_context(); }

uint64_t blasx_kernel_launch_count(void) { return bx::g_launches.load(); }

}  // extern "C"

extern "C" int blasx_test_fail_allocation(int nth) {
    bx::g_fail_alloc_countdown.store(nth > 0 ? nth : 0);
    return BLASX_OK;
}
