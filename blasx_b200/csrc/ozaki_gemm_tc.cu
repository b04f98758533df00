// ozaki_gemm_tc.cu -- the standalone INT8 residue GEMM launch: one persistent
// CTA per SM (or CTAs of bounded life when a launch asks for it), each
// running the tcgen05 pipeline of residue_tc.cuh over a strided walk of the
// output tiles, with the test hook that stalls one pipeline stage.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <mutex>

#include "ozaki.h"
#include "residue_tc.cuh"

namespace bx {
namespace oz {

namespace {

__global__ void __launch_bounds__(kThreadsTC, 1)
    residue_gemm_kernel(const __grid_constant__ CUtensorMap mapX,
                        const __grid_constant__ CUtensorMap mapY, const TcArgs a) {
    const int nmod = a.dec->nmod;
    const int tiles_j = a.tjn, tiles_i = int(a.Ip / kTileI);
    const int64_t total = int64_t(nmod) * tiles_j * tiles_i;
    if (total == 0) return;  // native fallback chosen on the device

    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const ResiduePipe p = residue_pipe_at(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) residue_pipe_init(p);
    if (warp == 1) tmem_alloc_all(p.tmem_slot);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *p.tmem_slot;

    // this CTA's tiles: a strided walk over the raster order
    TileSeq q;
    q.raster = true;
    q.first = blockIdx.x;
    q.step = gridDim.x;
    q.end = total;
    q.tiles_j = tiles_j;
    q.tiles_i = tiles_i;
    q.tj0 = a.tj0;
    q.tj = q.ti = 0;
    RolePos pos;
    residue_roles(&mapX, &mapY, a, q, seq_count(q, nmod), p, tmem, pos, warp, lane,
                  int(blockIdx.x) == a.stall_cta);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_free_all(tmem);
    }
}

// Test hook (blasx_test_stall_residue_gemm): the next g_stall_launches
// launches run with a wait limit of g_stall_wait cycles and CTA 0 issues no
// loads for its second pipeline stage.
std::atomic<int> g_stall_launches{0};
std::atomic<long long> g_stall_wait{kWaitCycles};

void take_stall(long long *wait_cycles, int *stall_cta) {
    if (take_residue_stall(wait_cycles)) *stall_cta = 0;
}

}  // namespace

bool take_residue_stall(long long *wait_cycles) {
    int n = g_stall_launches.load();
    while (n > 0) {
        if (g_stall_launches.compare_exchange_weak(n, n - 1)) {
            *wait_cycles = g_stall_wait.load();
            return true;
        }
    }
    return false;
}

int prepare_residue_gemm_current_device() {
    BX_CUDA(upload_moduli());
    BX_CUDA(cudaFuncSetAttribute(residue_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kSmemBytes)));
    return BLASX_OK;
}

int launch_residue_gemm(const int8_t *X, const int8_t *Y, uint8_t *U, int64_t Jp, int64_t Ip,
                        int64_t Kp, const Decision *dec, int *err_flag, int num_sms,
                        cudaStream_t s, int64_t tj_begin, int64_t tj_count, int max_cta_tiles, int uplo,
                        int64_t diag, int64_t jblock) {
    if (Jp % kTileJ || Ip % kTileI || Kp % kTileK || Kp > int64_t(kMaxK) * 2)
        return set_error(BLASX_ERR_UNSUPPORTED, "residue GEMM: bad padded extents");
    static std::once_flag once;
    static int init_status = BLASX_OK;
    std::call_once(once, [] {
        if (upload_moduli() != cudaSuccess ||
            cudaFuncSetAttribute(residue_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kSmemBytes)) != cudaSuccess)
            init_status = BLASX_ERR_CUDA;
    });
    if (init_status != BLASX_OK) return set_error(init_status, "residue GEMM init failed");
    CUtensorMap mx, my;
    BX_TRY(make_map(&mx, X, Jp, Kp, kTileJ));
    BX_TRY(make_map(&my, Y, Ip, Kp, kTileI));
    if (tj_count < 0) {
        tj_begin = 0;
        tj_count = Jp / kTileJ;
    }
    if (tj_begin < 0 || tj_begin + tj_count > Jp / kTileJ)
        return set_error(BLASX_ERR_ARG, "residue GEMM: j-tile range out of bounds");
    if (uplo && (jblock <= 0 || jblock % kTileJ || Jp % jblock))
        return set_error(BLASX_ERR_ARG, "residue GEMM: bad column block for a triangular output");
    TcArgs a{Jp, Ip, Kp, U, dec, err_flag, int(tj_begin), int(tj_count), uplo,
             uplo ? int(jblock / kTileJ) : 1, diag, kWaitCycles, -1};
    take_stall(&a.wait_cycles, &a.stall_cta);
    const int64_t tiles_upper = int64_t(kMaxModuli) * tj_count * (Ip / kTileI);
    if (tiles_upper == 0) return BLASX_OK;
    int64_t grid = tiles_upper < num_sms ? tiles_upper : num_sms;
    if (max_cta_tiles > 0) grid = std::max<int64_t>(grid, (tiles_upper + max_cta_tiles - 1) / max_cta_tiles);
    grid = std::min<int64_t>(grid, INT32_MAX);
    residue_gemm_kernel<<<unsigned(grid), kThreadsTC, kSmemBytes, s>>>(mx, my, a);
    BX_CUDA(cudaGetLastError());
    count_launch();
    return BLASX_OK;
}

}  // namespace oz
}  // namespace bx

extern "C" int blasx_test_stall_residue_gemm(int launches, long long wait_cycles) {
    if (launches < 0 || wait_cycles <= 0) return BLASX_ERR_ARG;
    bx::oz::g_stall_wait.store(wait_cycles);
    bx::oz::g_stall_launches.store(launches);
    return BLASX_OK;
}
