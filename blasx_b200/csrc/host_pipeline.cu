// host_pipeline.cu -- host-resident GEMM: copy operands into HBM, compute,
// copy C back.
//
// Replaces the reference's per-call flow of blas/dgemm.c:88-121 (pin A/B/C,
// build per-GPU caches, run the tiled runtime, unpin).
#include <chrono>

#include "host_pipeline.h"
#include "kernels.h"

namespace bx {

namespace {

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = nullptr;
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    int alloc(size_t bytes, cudaStream_t st) {
        s = st;
        BX_CUDA(cudaMallocAsync(&p, bytes ? bytes : 256, st));
        return BLASX_OK;
    }
};

}  // namespace

int host_gemm(const Gemm &g) {
    auto t0 = std::chrono::steady_clock::now();
    blasx_call_stats &st = call_stats();
    st = blasx_call_stats{};
    if (g.M == 0 || g.N == 0) return BLASX_OK;
    Context *c = context();
    if (!c) return last_status();
    std::lock_guard<std::mutex> lk(c->host_mu);
    cudaStream_t s = c->compute;
    const size_t es = elem_size(g.dt);
    const bool need_ab = !(g.alpha_zero() || g.K == 0);
    const bool read_c = !g.beta_zero();

    Gemm d = g;
    DevBuf bA, bB, bC;
    if (need_ab) {
        const int64_t lda = round_up(g.rows_a(), 32), ldb = round_up(g.rows_b(), 32);
        BX_TRY(bA.alloc(size_t(lda) * g.cols_a() * es, s));
        BX_TRY(bB.alloc(size_t(ldb) * g.cols_b() * es, s));
        BX_CUDA(cudaMemcpy2DAsync(bA.p, lda * es, g.A, g.lda * es, g.rows_a() * es, g.cols_a(),
                                  cudaMemcpyHostToDevice, s));
        BX_CUDA(cudaMemcpy2DAsync(bB.p, ldb * es, g.B, g.ldb * es, g.rows_b() * es, g.cols_b(),
                                  cudaMemcpyHostToDevice, s));
        d.A = bA.p; d.lda = lda;
        d.B = bB.p; d.ldb = ldb;
        st.h2d_bytes += double(es) * (g.rows_a() * g.cols_a() + g.rows_b() * g.cols_b());
    }
    const int64_t ldc = round_up(g.M, 32);
    BX_TRY(bC.alloc(size_t(ldc) * g.N * es, s));
    if (read_c) {
        BX_CUDA(cudaMemcpy2DAsync(bC.p, ldc * es, g.C, g.ldc * es, g.M * es, g.N,
                                  cudaMemcpyHostToDevice, s));
        st.h2d_bytes += double(es) * g.M * g.N;
    }
    d.C = bC.p; d.ldc = ldc;
    if (need_ab) {
        BX_TRY(device_gemm(d, s));
    } else {
        BX_TRY(launch_scale(d, s));
        st.path = 3;
    }
    BX_CUDA(cudaMemcpy2DAsync(g.C, g.ldc * es, bC.p, ldc * es, g.M * es, g.N,
                              cudaMemcpyDeviceToHost, s));
    st.d2h_bytes += double(es) * g.M * g.N;
    BX_CUDA(cudaStreamSynchronize(s));
    if (st.path == 2) {
        resolve_decision(st);
        if (*c->last_error_flag)
            return set_error(BLASX_ERR_TIMEOUT, "emulated GEMM: bounded device wait expired (flag %d)",
                             *c->last_error_flag);
    }
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return BLASX_OK;
}

}  // namespace bx
