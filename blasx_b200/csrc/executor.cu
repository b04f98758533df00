// executor.cu -- the serving loop's persistent tile executor (see executor.h).
//
// Device side: executor_kernel, one CTA of 256 threads per SM. Thread 0
// claims the next published task (a compare-and-swap on one device counter,
// after an acquire load of the ring's tail from pinned host memory, which
// also makes the task's inputs -- written by copies and by other CTAs before
// the task was published -- visible to the CTA's loads); the CTA copies the
// request's descriptor to shared memory, runs the task body, fences its
// writes to system scope and marks the task done in pinned host memory.
// Task bodies are the same device code as the standalone kernels:
//   kDmma     one C tile of a native FP64 (128x128) or complex128 (64x128)
//             request on the FP64 tensor pipe (dmma_tile.cuh)
//   kSimt     one C tile of a native FP32 (128x128) or complex64 (64x64)
//             request on the CUDA cores (simt_tile.cuh)
//   kScale    beta-scaling of a range of C (alpha == 0 or K == 0)
//   kZero     clearing of an emulated request's statistics and error word
//   kStats    row statistics of op(A) or op(B), a range of blocks
//   kDecide   the modulus count and norm bound (one CTA)
//   kSlice    int8 residues of op(A) or op(B), a range of blocks
//   kResidue  one 256 x 128 C tile for every modulus: the tcgen05 pipeline
//             of residue_tc.cuh, TMEM allocated once per CTA, its barriers
//             and ring positions carried from task to task
//   kRecon    CRT reconstruction and the alpha / beta epilogue, a range of
//             blocks (two 128-thread blocks at a time)
// Every wait is bounded: the claim gives up after idle_cycles without a task
// (or when the host raises the stop flag) and the CTA exits; the residue
// pipeline's mbarrier waits give up after their limit, raise the request's
// error word, and the pipeline is initialised again before the next task.
//
// Host side: the Executor owns the ring, the device descriptor table and the
// kernel's stream. Each request slot carries its list of stages; a stage's
// tasks are published when the previous stage has completed (for the
// emulated path the stage after the decision depends on it: the slices,
// residue tiles and reconstruction, or the native tiles when the device
// chose the native fallback).
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "dmma_tile.cuh"
#include "executor.h"
#include "kernels.h"
#include "ozaki_dev.cuh"
#include "residue_tc.cuh"
#include "simt_tile.cuh"

namespace bx {
namespace exec {

namespace {

using dev::DmmaParams;
using dev::SimtParams;

constexpr int kThreads = 256;
constexpr int64_t kRing = int64_t(1) << 16;  // task entries of each ring
// Two rings: lane 0 for requests of fewer than kFastFlops, lane 1 for the
// rest. A CTA always looks at lane 0 first, so that small requests do not
// wait behind the tiles of large ones.
constexpr int kLanes = 2;
constexpr double kFastFlops = 2e9;
// The kernel's CTAs stay while the host keeps it running and leave together
// when the host raises the stop flag (kLinger without work). A CTA that sees
// no task for kIdleCycles makes them all leave: a bound for the case of a
// host that stopped publishing without stopping the kernel. The host
// launches the kernel again when tasks are pending and it has ended.
constexpr long long kIdleCycles = 400000000;  // ~0.2 s
constexpr double kLinger = 0.005;             // s without pending tasks before the host stops the kernel

enum Kind : int32_t {
    kNone = 0,
    kZero,
    kStats,
    kDecide,
    kSlice,
    kResidue,
    kRecon,
    kDmma,
    kSimt,
    kScale,
};

struct Task {
    int32_t kind, slot, side, stall;  // side: 0 op(A), 1 op(B); stall: test hook
    int64_t first, count;             // units of the kind: blocks, tiles or elements
    long long wait;                   // residue pipeline wait limit (clock cycles)
    int64_t pad;
};
static_assert(sizeof(Task) == 48, "task layout");

// Everything a task of one request needs, built on the host, copied to the
// device table before the request's first task is published.
struct alignas(128) ReqDesc {
    CUtensorMap mapX, mapY;  // residue GEMM operands (128-byte aligned)
    int dt, emulated, akc, bkc;
    int alias, mode, forced, rc_blocks_a;
    double unit;
    // native
    DmmaParams dp;
    SimtParams<float> sf;
    SimtParams<c2> sc;
    SimtParams<double> sd;  // scale only
    SimtParams<z2> sz;      // scale only
    int64_t simt_tm;        // SIMT tiles along M
    int64_t simt_edge;      // SIMT tile edge: 128 (FP32) or 64 (complex64)
    // emulated
    oz::View va, vb;
    oz::RowStats sa, sb, sbd;
    oz::Decision *dec;
    int *ea, *fb, *err;
    oz::SliceOut oy, ox;
    int64_t M, N, K, Kc;
    uint32_t *zero_ptr;
    int64_t zero_words;
    int64_t stats_gx[2], slice_gx[2], recon_gx;
    int64_t res_tiles_j, res_tiles_i;
    oz::TcArgs tc;
    oz::ReconArgs ra;
};
static_assert(sizeof(ReqDesc) % 16 == 0, "descriptor copied in 16-byte words");

struct ExecArgs {
    const Task *ring[kLanes];               // pinned host, device view
    volatile uint32_t *done[kLanes];        // pinned host: task i done <=> done[i % kRing] == i + 1
    const volatile long long *tail[kLanes]; // pinned host: tasks published
    const volatile int *stop;               // pinned host: exit at the next claim
    volatile int *err_host;                 // pinned host, per slot: device error word seen
    oz::Decision *dec_host;                 // pinned host, per slot: the decision
    unsigned long long *next;               // device, per lane: next task to claim
    long long *dev_tail;                    // device, per lane: tasks known to be published
    unsigned *poll_lock;              // device: one CTA at a time reads the host's tail
    int *dev_stop;                    // device: the host's stop flag was seen
    const ReqDesc *descs;             // device, per slot
    unsigned long long *tasks_run;    // device counter
    long long idle_cycles;
};

// Shared memory: a 1024-byte aligned work area that every task kind uses in
// turn (DMMA operand stages, SIMT k-steps, the slice transpose, the residue
// ring), with the alignment slack.
constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t kWorkBytes = cmax(
    cmax(cmax(dev::dmma_smem_bytes<false, true, true>(), dev::dmma_smem_bytes<false, true, false>()),
         cmax(dev::dmma_smem_bytes<false, false, true>(), dev::dmma_smem_bytes<false, false, false>())),
    cmax(cmax(cmax(dev::dmma_smem_bytes<true, true, true>(), dev::dmma_smem_bytes<true, true, false>()),
              cmax(dev::dmma_smem_bytes<true, false, true>(), dev::dmma_smem_bytes<true, false, false>())),
         cmax(oz::kRingBytes, cmax(oz::slice_rc_smem_bytes<1>(),
                                   cmax(dev::simt_smem_bytes<c2>(), dev::sgemm128_smem_bytes())))));
constexpr size_t kDynSmem = kWorkBytes + 1024;

__device__ __forceinline__ long long ld_acquire_sys(const volatile long long *p) {
    long long v;
    asm volatile("ld.acquire.sys.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire_sys(const volatile int *p) {
    int v;
    asm volatile("ld.acquire.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_gpu(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_sys(volatile uint32_t *p, uint32_t v) {
    asm volatile("st.release.sys.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ long long ld_acquire_gpu(const long long *p) {
    long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void max_release_gpu(long long *p, long long v) {
    asm volatile("red.release.gpu.global.max.s64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Claims the next published task (thread 0), lane 0 first. False once a
// stop was seen (the host's flag, or a CTA that found no task for
// idle_cycles): then every CTA leaves at its next claim. The tasks known to be
// published are mirrored in device memory (dev_tail): the CTAs poll that,
// and only when it shows nothing new does one of them at a time (poll_lock)
// read the host's tails and stop flag across PCIe, with a growing pause
// between looks while the rings stay empty.
__device__ bool claim(const ExecArgs &a, Task *task, long long *index, int *lane) {
    const long long t0 = clock64();
    unsigned pause = 64;  // ns
    for (;;) {
        // a stop, once seen by any CTA, ends every CTA at its next claim,
        // tasks left or not: the kernel then ends as a whole and the host
        // launches it again for what is pending (a kernel that went on with
        // the CTAs that still found tasks would look live to the host with a
        // fraction of the SMs)
        if (*reinterpret_cast<volatile int *>(a.dev_stop)) return false;
        bool known = false;
#pragma unroll 1
        for (int l = 0; l < kLanes; ++l) {
            const long long tail = ld_acquire_gpu(a.dev_tail + l);
            const unsigned long long i = ld_relaxed_gpu(a.next + l);
            if (static_cast<long long>(i) >= tail) continue;
            known = true;
            if (atomicCAS(a.next + l, i, i + 1) != i) break;  // lost the race: look again from lane 0
            const volatile int4 *src = reinterpret_cast<const volatile int4 *>(a.ring[l] + (i % kRing));
            int4 v[sizeof(Task) / 16];
#pragma unroll
            for (int w = 0; w < int(sizeof(Task) / 16); ++w) v[w] = {src[w].x, src[w].y, src[w].z, src[w].w};
            int4 *dst = reinterpret_cast<int4 *>(task);
#pragma unroll
            for (int w = 0; w < int(sizeof(Task) / 16); ++w) dst[w] = v[w];
            *index = static_cast<long long>(i);
            *lane = l;
            // what the task reads was written before it was published: order
            // the CTA's coming loads after that (no stale cached lines)
            asm volatile("fence.acq_rel.gpu;" ::: "memory");
            return true;
        }
        if (known) {
            pause = 64;
            continue;
        }
        if (atomicCAS(a.poll_lock, 0u, 1u) == 0u) {
            const int stop = ld_acquire_sys(a.stop);
            bool more = false;
#pragma unroll 1
            for (int l = 0; l < kLanes; ++l) {
                const long long host_tail = ld_acquire_sys(a.tail[l]);
                if (host_tail > ld_acquire_gpu(a.dev_tail + l)) {
                    max_release_gpu(a.dev_tail + l, host_tail);
                    more = true;
                }
            }
            if (stop) atomicExch(a.dev_stop, 1);
            atomicExch(a.poll_lock, 0u);
            if (more) {
                pause = 64;
                continue;
            }
        }
        if (*reinterpret_cast<volatile int *>(a.dev_stop)) return false;
        if (clock64() - t0 > a.idle_cycles) {  // the whole kernel leaves, not this CTA alone
            atomicExch(a.dev_stop, 1);
            return false;
        }
        __nanosleep(pause);
        if (pause < 8192) pause *= 2;
    }
}

template <typename T> struct Scale;
template <> struct Scale<float> { __device__ static const SimtParams<float> &of(const ReqDesc &d) { return d.sf; } };
template <> struct Scale<double> { __device__ static const SimtParams<double> &of(const ReqDesc &d) { return d.sd; } };
template <> struct Scale<c2> { __device__ static const SimtParams<c2> &of(const ReqDesc &d) { return d.sc; } };
template <> struct Scale<z2> { __device__ static const SimtParams<z2> &of(const ReqDesc &d) { return d.sz; } };

template <typename S>
__device__ __forceinline__ void scale_task(const ReqDesc &d, const Task &t, int tid) {
    const SimtParams<S> &p = Scale<S>::of(d);
    dev::scale_range<S>(p.M, p.beta, p.C, p.ldc, p.beta_zero, p.uplo, p.diag, t.first + tid, t.first + t.count,
                        kThreads);
}

// The emulated stages for element type T (double, float, zpair, cpair).
template <typename T>
__device__ __forceinline__ void emulated_task(const ReqDesc &d, const Task &t, int tid, uint8_t *work) {
    constexpr bool CPLX = oz::Elem<T>::cplx;
    const int side = t.side;
    switch (t.kind) {
        case kStats: {
            const oz::View &v = side ? d.vb : d.va;
            const oz::RowStats &st = side ? d.sb : d.sa;
            const bool kc = side ? d.bkc : d.akc;
            for (int64_t b = t.first; b < t.first + t.count; ++b) {
                if (kc) oz::stats_kc_body<T>(v, st, b, tid);
                else oz::stats_rc_body<T>(v, st, 512, b % d.stats_gx[side], b / d.stats_gx[side], tid);
            }
            break;
        }
        case kSlice: {
            const oz::View &v = side ? d.vb : d.va;
            const oz::RowStats &st = side ? d.sb : d.sa;
            const oz::SliceOut &o = side ? d.ox : d.oy;
            int *expo = side ? d.fb : d.ea;
            const bool kc = side ? d.bkc : d.akc;
            const int64_t gx = d.slice_gx[side];
            for (int64_t b = t.first; b < t.first + t.count; ++b) {
                if constexpr (CPLX) {
                    if (side == 0) {
                        if (kc) oz::slice_kc_body<T, 1>(v, st, d.dec, expo, o, b % gx, b / gx, tid);
                        else oz::slice_rc_body<T, 1>(v, st, d.dec, expo, o, b % gx, b / gx, tid, work);
                    } else {
                        if (kc) oz::slice_kc_body<T, 2>(v, st, d.dec, expo, o, b % gx, b / gx, tid);
                        else oz::slice_rc_body<T, 2>(v, st, d.dec, expo, o, b % gx, b / gx, tid, work);
                    }
                } else {
                    if (kc) oz::slice_kc_body<T, 0>(v, st, d.dec, expo, o, b % gx, b / gx, tid);
                    else oz::slice_rc_body<T, 0>(v, st, d.dec, expo, o, b % gx, b / gx, tid, work);
                }
                if (!kc) __syncthreads();  // the transpose tile is reused by the next block
            }
            break;
        }
        case kRecon: {
            // two 128-thread blocks at a time
            const int half = tid >> 7, ht = tid & 127;
            for (int64_t b = t.first + half; b < t.first + t.count; b += 2)
                oz::reconstruct_body<T, CPLX>(d.ra, d.dec, b % d.recon_gx, b / d.recon_gx, ht);
            break;
        }
        default:
            break;
    }
}

// Not inlined: the tile's accumulators get the registers that the
// executor's own loop state would otherwise take from them.
template <bool CPLX, int KI>
__device__ __noinline__ void dmma_task(const ReqDesc &d, const Task &t, uint8_t *work) {
    double *smem = reinterpret_cast<double *>(work);
    for (int64_t tile = t.first; tile < t.first + t.count; ++tile) {
        if (d.akc) {
            if (d.bkc) dev::dmma_tile<CPLX, true, true, KI>(d.dp, int(tile), smem);
            else dev::dmma_tile<CPLX, true, false, KI>(d.dp, int(tile), smem);
        } else {
            if (d.bkc) dev::dmma_tile<CPLX, false, true, KI>(d.dp, int(tile), smem);
            else dev::dmma_tile<CPLX, false, false, KI>(d.dp, int(tile), smem);
        }
        __syncthreads();  // the stages are reused by the next tile
    }
}

template <typename T>
__device__ __forceinline__ void simt_task(const SimtParams<T> &p, int64_t tm, const Task &t, uint8_t *work) {
    for (int64_t tile = t.first; tile < t.first + t.count; ++tile) {
        dev::simt_tile<T>(p, tile % tm, tile / tm, reinterpret_cast<T *>(work));
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads, 1) executor_kernel(const ExecArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *work = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ uint64_t s_bars[2 * oz::kStages + 5];
    __shared__ uint32_t s_tmem_slot;
    __shared__ int s_abort;
    __shared__ Task s_task;
    __shared__ long long s_index;
    __shared__ int s_lane;
    __shared__ ReqDesc s_desc;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // the residue pipeline: its ring is the work area, its barriers live apart
    oz::ResiduePipe pipe;
    pipe.ring = work;
    pipe.full0 = oz::su32(s_bars);
    pipe.empty0 = oz::su32(s_bars + oz::kStages);
    pipe.tfull0 = oz::su32(s_bars + 2 * oz::kStages);
    pipe.tempty0 = oz::su32(s_bars + 2 * oz::kStages + 2);
    pipe.done = oz::su32(s_bars + 2 * oz::kStages + 4);
    pipe.tmem_slot = &s_tmem_slot;
    pipe.abort_flag = &s_abort;
    if (tid == 0) oz::residue_pipe_init(pipe);
    if (warp == 1) oz::tmem_alloc_all(pipe.tmem_slot);
    oz::tc_fence_before();
    __syncthreads();
    oz::tc_fence_after();
    const uint32_t tmem = s_tmem_slot;
    oz::RolePos pos;

    for (;;) {
        if (tid == 0) {
            Task t;
            long long i = 0;
            int lane = 0;
            if (!claim(a, &t, &i, &lane)) t.kind = kNone;
            s_task = t;
            s_index = i;
            s_lane = lane;
        }
        __syncthreads();
        const Task t = s_task;
        if (t.kind == kNone) break;
        // the request's descriptor, through L2
        {
            const uint4 *src = reinterpret_cast<const uint4 *>(a.descs + t.slot);
            uint4 *dst = reinterpret_cast<uint4 *>(&s_desc);
            for (int w = tid; w < int(sizeof(ReqDesc) / 16); w += kThreads) dst[w] = __ldcg(src + w);
        }
        __syncthreads();
        const ReqDesc &d = s_desc;
        const DType dt = DType(d.dt);
        switch (t.kind) {
            case kZero:
                for (int64_t w = t.first + tid; w < t.first + t.count; w += kThreads) d.zero_ptr[w] = 0u;
                break;
            case kDecide:
                oz::decide_body(d.sa, d.M, d.sbd, d.N, d.K, d.unit, d.mode, d.forced, d.dec, tid, kThreads);
                break;
            case kStats:
            case kSlice:
            case kRecon:
                if (dt == DType::F64) emulated_task<double>(d, t, tid, work);
                else if (dt == DType::F32) emulated_task<float>(d, t, tid, work);
                else if (dt == DType::C128) emulated_task<oz::zpair>(d, t, tid, work);
                else emulated_task<oz::cpair>(d, t, tid, work);
                break;
            case kResidue: {
                const int nmod = __ldcg(&d.dec->nmod);
                if (nmod > 0) {
                    const oz::TileCoord c = oz::decode(t.first, int(d.res_tiles_j), int(d.res_tiles_i), 0);
                    oz::TileSeq q;
                    q.raster = false;
                    q.first = q.step = q.end = 0;
                    q.tiles_j = q.tiles_i = q.tj0 = 0;
                    q.tj = c.tj;
                    q.ti = c.ti;
                    oz::TcArgs ta = d.tc;
                    ta.wait_cycles = t.wait;
                    const CUtensorMap *mx = &a.descs[t.slot].mapX, *my = &a.descs[t.slot].mapY;
                    if (warp == 0 && lane == 0) {
                        // the maps and the slices were written by the generic proxy
                        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mx) : "memory");
                        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(my) : "memory");
                        asm volatile("fence.proxy.async.global;" ::: "memory");
                    }
                    oz::residue_roles(mx, my, ta, q, nmod, pipe, tmem, pos, warp, lane, t.stall != 0);
                }
                break;
            }
            case kDmma:
                if (dt == DType::C128) dmma_task<true, 4>(d, t, work);
                else dmma_task<false, 16>(d, t, work);
                break;
            case kSimt:
                if (dt == DType::F32) {
                    for (int64_t tile = t.first; tile < t.first + t.count; ++tile) {
                        dev::sgemm128_tile(d.sf, tile % d.simt_tm, tile / d.simt_tm, reinterpret_cast<float *>(work));
                        __syncthreads();
                    }
                } else {
                    simt_task<c2>(d.sc, d.simt_tm, t, work);
                }
                break;
            case kScale:
                if (dt == DType::F32) scale_task<float>(d, t, tid);
                else if (dt == DType::F64) scale_task<double>(d, t, tid);
                else if (dt == DType::C64) scale_task<c2>(d, t, tid);
                else scale_task<z2>(d, t, tid);
                break;
            default:
                break;
        }
        oz::tc_fence_before();
        __syncthreads();  // the task's writes, ordered before thread 0's system fence below
        oz::tc_fence_after();
        if (s_abort) {
            // a residue pipeline gave up; its copies and MMAs have drained, so
            // its barriers can be initialised again
            __syncthreads();
            if (tid == 0) oz::residue_pipe_init(pipe);
            pos = oz::RolePos{};
            __syncthreads();
        }
        if (tid == 0) {
            if (t.kind == kDecide) {
                const oz::Decision dd = *d.dec;  // written by this CTA
                a.dec_host[t.slot] = dd;
            }
            if (t.kind == kResidue && d.err) {
                const int e = __ldcg(d.err);
                if (e) a.err_host[t.slot] = e;
            }
            __threadfence_system();
            st_release_sys(a.done[s_lane] + (s_index % kRing), uint32_t(s_index + 1));
            atomicAdd(a.tasks_run, 1ull);
        }
    }
    oz::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        oz::tc_fence_after();
        oz::tmem_free_all(tmem);
    }
}

// ---- host side -------------------------------------------------------------------

struct Stage {
    std::vector<Task> tasks;
};

struct Slot {
    bool active = false;
    bool emulated = false;
    int dt = 0;
    std::vector<Stage> stages;    // published in order
    std::vector<Stage> fallback;  // emulated: replaces the stages after the decision when nmod == 0
    int decide_stage = -1;        // index of the decision stage (emulated)
    int stage = -1;               // current stage
    long long first = 0, count = 0, scan = 0;  // ring indices of the current stage, first not yet seen done
    int lane = 1;                 // its ring
    int path = 0, moduli = 0;
};

struct Lane {
    Task *ring = nullptr;             // pinned host
    volatile uint32_t *done = nullptr;
    volatile long long *tail = nullptr;
    long long published = 0, floor = 0;  // tasks published / first not seen done
    bool is_done(long long i) const { return done[i % kRing] == uint32_t(i + 1); }
};

}  // namespace

class Executor {
public:
    int slots = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_end = nullptr;
    bool launched = false;
    // pinned host
    Lane lanes[kLanes];
    volatile int *stop_flag = nullptr;
    volatile int *err_host = nullptr;
    oz::Decision *dec_host = nullptr;
    ReqDesc *staging = nullptr;  // per slot, source of the descriptor copies
    void *host_words = nullptr;  // the tails and the stop flag
    // device
    unsigned long long *next = nullptr;  // per lane, then the task counter, tails, lock and stop word
    unsigned long long *tasks_run = nullptr;
    ReqDesc *descs = nullptr;
    long long launches = 0;
    std::vector<Slot> state;

    bool stopping = false;       // the stop flag is raised; the kernel is draining
    double idle_since = -1.0;    // when the last pending task completed (s), -1 while tasks are pending
    bool running() {
        if (!launched) return false;
        const cudaError_t q = cudaEventQuery(ev_end);
        if (q == cudaErrorNotReady) return true;
        if (q != cudaSuccess) cudaGetLastError();
        launched = false;
        if (stopping) {
            *stop_flag = 0;
            stopping = false;
        }
        return false;
    }
    static double now_s() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }
    int launch() {
        ExecArgs a;
        void *p = nullptr;
        for (int l = 0; l < kLanes; ++l) {
            BX_CUDA(cudaHostGetDevicePointer(&p, lanes[l].ring, 0));
            a.ring[l] = static_cast<const Task *>(p);
            BX_CUDA(cudaHostGetDevicePointer(&p, const_cast<uint32_t *>(lanes[l].done), 0));
            a.done[l] = static_cast<volatile uint32_t *>(p);
            BX_CUDA(cudaHostGetDevicePointer(&p, const_cast<long long *>(lanes[l].tail), 0));
            a.tail[l] = static_cast<const volatile long long *>(p);
        }
        BX_CUDA(cudaHostGetDevicePointer(&p, const_cast<int *>(stop_flag), 0));
        a.stop = static_cast<const volatile int *>(p);
        BX_CUDA(cudaHostGetDevicePointer(&p, const_cast<int *>(err_host), 0));
        a.err_host = static_cast<volatile int *>(p);
        BX_CUDA(cudaHostGetDevicePointer(&p, dec_host, 0));
        a.dec_host = static_cast<oz::Decision *>(p);
        a.next = next;  // next[0..kLanes)
        a.tasks_run = tasks_run;
        a.dev_tail = reinterpret_cast<long long *>(next + kLanes + 1);
        a.poll_lock = reinterpret_cast<unsigned *>(next + 2 * kLanes + 1);
        a.dev_stop = reinterpret_cast<int *>(next + 2 * kLanes + 2);
        a.descs = descs;
        a.idle_cycles = kIdleCycles;
        *stop_flag = 0;
        stopping = false;
        BX_CUDA(cudaMemsetAsync(a.poll_lock, 0, 2 * sizeof(unsigned long long), stream));  // lock and stop word
        executor_kernel<<<unsigned(num_sms), kThreads, kDynSmem, stream>>>(a);
        BX_CUDA(cudaGetLastError());
        count_launch();
        BX_CUDA(cudaEventRecord(ev_end, stream));
        launched = true;
        ++launches;
        return BLASX_OK;
    }
    // Entry i of a ring is free once its task i - kRing is done.
    int publish(int l, const Task &t) {
        Lane &ln = lanes[l];
        const long long i = ln.published;
        while (i >= kRing && !ln.is_done(i - kRing)) {
            BX_TRY(pump_kernel());
            std::this_thread::yield();
        }
        ln.ring[i % kRing] = t;
        std::atomic_thread_fence(std::memory_order_release);
        *ln.tail = i + 1;
        ln.published = i + 1;
        return BLASX_OK;
    }
    bool pending() {
        bool any = false;
        for (Lane &ln : lanes) {
            while (ln.floor < ln.published && ln.is_done(ln.floor)) ++ln.floor;
            any = any || ln.floor < ln.published;
        }
        return any;
    }
    // Launches the kernel when tasks are pending and it is not running; stops
    // it (without waiting) once nothing has been pending for kLinger.
    int pump_kernel() {
        const bool busy = pending();
        const bool live = running();
        if (busy) {
            idle_since = -1.0;
            if (!live) BX_TRY(launch());
        } else if (live && !stopping) {
            const double t = now_s();
            if (idle_since < 0) idle_since = t;
            else if (t - idle_since > kLinger) {
                *stop_flag = 1;
                std::atomic_thread_fence(std::memory_order_seq_cst);
                stopping = true;
            }
        }
        return BLASX_OK;
    }
    int publish_stage(int slot, int k) {
        Slot &sl = state[size_t(slot)];
        sl.stage = k;
        sl.first = lanes[sl.lane].published;
        sl.count = int64_t(sl.stages[size_t(k)].tasks.size());
        sl.scan = sl.first;
        for (Task t : sl.stages[size_t(k)].tasks) {
            if (t.kind == kResidue) {
                long long w = 0;
                if (oz::take_residue_stall(&w)) {
                    t.stall = 1;
                    t.wait = w;
                }
            }
            BX_TRY(publish(sl.lane, t));
        }
        return pump_kernel();
    }
};

namespace {

constexpr long long kDefaultWait = 2000000000LL;  // residue waits: ~1 s at 1.9 GHz

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Units per task for an elementwise stage: about four tasks per SM, so that
// a stage spreads over the whole GPU, with at least min_per units per task.
int64_t spread(int64_t units, int64_t min_per, int num_sms) {
    return std::max<int64_t>(min_per, cdiv(units, 4 * int64_t(std::max(1, num_sms))));
}

// Tasks of `units` units, `per` units each.
void add_tasks(Stage &st, int kind, int slot, int side, int64_t units, int64_t per) {
    per = std::max<int64_t>(1, per);
    for (int64_t f = 0; f < units; f += per) {
        Task t{};
        t.kind = kind;
        t.slot = slot;
        t.side = side;
        t.first = f;
        t.count = std::min(per, units - f);
        t.wait = kDefaultWait;
        st.tasks.push_back(t);
    }
}

template <typename T> SimtParams<T> simt_params(const Gemm &g) {
    return SimtParams<T>{g.ta, g.tb, int(g.M), int(g.N), int(g.K), from_cplx<T>(g.alpha), from_cplx<T>(g.beta),
                         static_cast<const T *>(g.A), g.lda, static_cast<const T *>(g.B), g.ldb,
                         static_cast<T *>(g.C), g.ldc, g.beta_zero() ? 1 : 0, g.uplo, g.diag};
}

// The native tiles of g: DMMA for FP64 / complex128, SIMT for FP32 / complex64.
Stage native_stage(ReqDesc &d, const Gemm &g, int slot) {
    Stage st;
    if (g.dt == DType::F64 || g.dt == DType::C128) {
        d.dp = g.dt == DType::F64 ? dev::make_params<false, 0>(g) : dev::make_params<true, 0>(g);
        add_tasks(st, kDmma, slot, 0, int64_t(d.dp.tiles_m) * d.dp.tiles_n, 1);
    } else {
        // FP32 on the 128 x 128 tile, complex64 on the 64 x 64 one
        if (g.dt == DType::F32) d.sf = simt_params<float>(g);
        else d.sc = simt_params<c2>(g);
        d.simt_edge = g.dt == DType::F32 ? dev::sg::TM : dev::kSimtBM;
        d.simt_tm = cdiv(g.M, d.simt_edge);
        add_tasks(st, kSimt, slot, 0, d.simt_tm * cdiv(g.N, d.simt_edge), 1);
    }
    return st;
}

}  // namespace

int create(int slots, Executor **out) {
    *out = nullptr;
    auto *e = new Executor;
    e->slots = slots;
    e->state.assign(size_t(slots), Slot{});
    auto fail = [&](int rc) {
        destroy(e);
        return rc;
    };
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return fail(set_error(BLASX_ERR_CUDA, "executor: device query failed"));
    auto host = [&](void **p, size_t bytes, unsigned flags) {
        if (cudaHostAlloc(p, bytes, flags) != cudaSuccess) return false;
        memset(*p, 0, bytes);
        return true;
    };
    void *p = nullptr;
    for (int l = 0; l < kLanes; ++l) {
        if (!host(&p, size_t(kRing) * sizeof(Task), cudaHostAllocMapped))
            return fail(set_error(BLASX_ERR_NOMEM, "executor: ring"));
        e->lanes[l].ring = static_cast<Task *>(p);
        if (!host(&p, size_t(kRing) * sizeof(uint32_t), cudaHostAllocMapped))
            return fail(set_error(BLASX_ERR_NOMEM, "executor: done flags"));
        e->lanes[l].done = static_cast<volatile uint32_t *>(p);
    }
    if (!host(&p, 256, cudaHostAllocMapped)) return fail(set_error(BLASX_ERR_NOMEM, "executor: tails"));
    e->host_words = p;
    for (int l = 0; l < kLanes; ++l)
        e->lanes[l].tail = reinterpret_cast<volatile long long *>(static_cast<char *>(p) + 64 * l);
    e->stop_flag = reinterpret_cast<volatile int *>(static_cast<char *>(p) + 64 * kLanes);
    if (!host(&p, sizeof(int) * size_t(slots), cudaHostAllocMapped)) return fail(set_error(BLASX_ERR_NOMEM, "executor: error words"));
    e->err_host = static_cast<volatile int *>(p);
    if (!host(&p, sizeof(oz::Decision) * size_t(slots), cudaHostAllocMapped)) return fail(set_error(BLASX_ERR_NOMEM, "executor: decisions"));
    e->dec_host = static_cast<oz::Decision *>(p);
    if (!host(&p, sizeof(ReqDesc) * size_t(slots), cudaHostAllocDefault)) return fail(set_error(BLASX_ERR_NOMEM, "executor: staging"));
    e->staging = static_cast<ReqDesc *>(p);
    if (dev_malloc(reinterpret_cast<void **>(&e->next), 256) != cudaSuccess ||
        dev_malloc(reinterpret_cast<void **>(&e->descs), sizeof(ReqDesc) * size_t(slots)) != cudaSuccess) {
        cudaGetLastError();
        return fail(set_error(BLASX_ERR_NOMEM, "executor: device tables"));
    }
    e->tasks_run = e->next + kLanes;
    if (cudaMemset(e->next, 0, 256) != cudaSuccess ||
        cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_end, cudaEventDisableTiming) != cudaSuccess ||
        cudaFuncSetAttribute(executor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kDynSmem)) !=
            cudaSuccess ||
        oz::upload_tables() != cudaSuccess || oz::upload_moduli() != cudaSuccess) {
        cudaGetLastError();
        return fail(set_error(BLASX_ERR_CUDA, "executor: set-up failed"));
    }
    *out = e;
    return BLASX_OK;
}

void destroy(Executor *e) {
    if (!e) return;
    if (e->stream) stop(e);
    if (e->ev_end) cudaEventDestroy(e->ev_end);
    if (e->stream) cudaStreamDestroy(e->stream);
    if (e->next) cudaFree(e->next);
    if (e->descs) cudaFree(e->descs);
    for (Lane &ln : e->lanes) {
        if (ln.ring) cudaFreeHost(ln.ring);
        if (ln.done) cudaFreeHost(const_cast<uint32_t *>(ln.done));
    }
    if (e->host_words) cudaFreeHost(e->host_words);
    if (e->err_host) cudaFreeHost(const_cast<int *>(e->err_host));
    if (e->dec_host) cudaFreeHost(e->dec_host);
    if (e->staging) cudaFreeHost(e->staging);
    delete e;
}

bool supports(const Gemm &g) { return g.a_form == kGeneral && g.b_form == kGeneral && !g.herm_out; }

int prepare(Executor *e, int slot, const Gemm &g, bool emulated, int mode, void *ws, cudaStream_t s) {
    if (slot < 0 || slot >= e->slots) return set_error(BLASX_ERR_ARG, "executor: slot %d", slot);
    Slot &sl = e->state[size_t(slot)];
    sl = Slot{};
    sl.active = true;
    sl.dt = int(g.dt);
    sl.lane = g.flops() < kFastFlops ? 0 : 1;
    ReqDesc &d = e->staging[slot];
    memset(static_cast<void *>(&d), 0, sizeof d);
    d.dt = int(g.dt);
    d.akc = g.ta != NoTrans;
    d.bkc = g.tb == NoTrans;
    const bool need_ab = !(g.alpha_zero() || g.K == 0);
    if (!need_ab) {
        switch (g.dt) {
            case DType::F32: d.sf = simt_params<float>(g); break;
            case DType::F64: d.sd = simt_params<double>(g); break;
            case DType::C64: d.sc = simt_params<c2>(g); break;
            default: d.sz = simt_params<z2>(g); break;
        }
        Stage st;
        add_tasks(st, kScale, slot, 0, g.M * g.N, spread(g.M * g.N, 1 << 15, e->num_sms));
        sl.stages.push_back(st);
        sl.path = 1;
    } else if (!emulated) {
        sl.stages.push_back(native_stage(d, g, slot));
        sl.path = 1;
    } else {
        sl.emulated = true;
        d.emulated = 1;
        const bool cplx = is_complex(g.dt);
        const oz::Plan pl = oz::make_plan(g);
        const oz::Parts pt = oz::carve_parts(g, pl, ws);
        d.va = oz::View{g.A, g.lda, pl.M, pl.K, g.ta == ConjT};
        d.vb = oz::View{g.B, g.ldb, pl.N, pl.K, g.tb == ConjT};
        d.sa = pt.sa;
        d.sb = pt.sb;
        d.sbd = pl.alias ? pt.sa : pt.sb;
        d.dec = pt.dec;
        d.ea = pt.ea;
        d.fb = pt.fb;
        d.err = pt.err;
        d.alias = pl.alias;
        d.mode = mode;
        d.forced = oz::forced_moduli();
        const bool single = g.dt == DType::F32 || g.dt == DType::C64;
        d.unit = single ? std::ldexp(1.0, -24) : std::ldexp(1.0, -53);
        d.M = pl.M;
        d.N = pl.N;
        d.K = pl.K;
        d.Kc = pl.Kc;
        d.oy = oz::SliceOut{pt.Y, pl.Ip, pl.Kp, pl.Kh, pl.Ip * pl.Kp};
        d.ox = oz::SliceOut{pt.X, pl.Jp, pl.Kp, pl.Kh, pl.Jx * pl.Kp};
        // the error word, the decision and the statistics, contiguous from the scratch's start
        d.zero_ptr = reinterpret_cast<uint32_t *>(pt.err);
        d.zero_words = int64_t((reinterpret_cast<char *>(pt.ea) - reinterpret_cast<char *>(pt.err)) / 4);
        Stage zero, stats, decide, slice, residue, recon;
        add_tasks(zero, kZero, slot, 0, d.zero_words, spread(d.zero_words, 1 << 14, e->num_sms));
        for (int side = 0; side < (pl.alias ? 1 : 2); ++side) {
            const int64_t R = side ? pl.N : pl.M;
            const bool kc = side ? d.bkc : d.akc;
            if (kc) {
                add_tasks(stats, kStats, slot, side, cdiv(R, 8), spread(cdiv(R, 8), 1, e->num_sms));
            } else {
                d.stats_gx[side] = cdiv(R, 256);
                const int64_t blocks = d.stats_gx[side] * cdiv(pl.K, 512);
                add_tasks(stats, kStats, slot, side, blocks, spread(blocks, 1, e->num_sms));
            }
            const int64_t Rp = side ? pl.Jp : pl.Ip;
            const int64_t kt = (kc || !cplx) ? 64 : 32;
            d.slice_gx[side] = pl.Kc / kt;
            const int64_t blocks = d.slice_gx[side] * (Rp / 64);
            add_tasks(slice, kSlice, slot, side, blocks, spread(blocks, 1, e->num_sms));
        }
        add_tasks(decide, kDecide, slot, 0, 1, 1);
        d.res_tiles_j = pl.Jx / oz::kTileJ;
        d.res_tiles_i = pl.Ip / oz::kTileI;
        d.tc = oz::TcArgs{pl.Jx, pl.Ip, pl.Kp, pt.U, pt.dec, pt.err, 0, int(d.res_tiles_j), g.uplo,
                          g.uplo ? int(pl.Jp / oz::kTileJ) : 1, g.diag, kDefaultWait, -1};
        add_tasks(residue, kResidue, slot, 0, d.res_tiles_j * d.res_tiles_i, 1);
        BX_TRY(oz::make_map(&d.mapX, pt.X, pl.Jx, pl.Kp, oz::kTileJ));
        BX_TRY(oz::make_map(&d.mapY, pt.Y, pl.Ip, pl.Kp, oz::kTileI));
        d.ra = oz::ReconArgs{pt.U, pl.Jp, pl.Ip, pl.M, pl.N, pt.ea, pl.alias ? pt.ea : pt.fb, g.alpha.re, g.alpha.im,
                             g.beta.re, g.beta.im, g.beta_zero() ? 1 : 0, g.C, g.ldc, 0, g.uplo, g.diag};
        d.recon_gx = cdiv(pl.M, 512);
        add_tasks(recon, kRecon, slot, 0, d.recon_gx * pl.N, spread(d.recon_gx * pl.N, 8, e->num_sms));
        sl.stages = {zero, stats, decide, slice, residue, recon};
        sl.decide_stage = 2;
        sl.fallback.push_back(native_stage(d, g, slot));
        sl.path = 2;
    }
    BX_CUDA(cudaMemcpyAsync(e->descs + slot, &d, sizeof d, cudaMemcpyHostToDevice, s));
    return BLASX_OK;
}

int start(Executor *e, int slot) {
    Slot &sl = e->state[size_t(slot)];
    e->err_host[slot] = 0;
    e->dec_host[slot].nmod = -1;
    if (sl.stages.empty()) return BLASX_OK;
    return e->publish_stage(slot, 0);
}

int advance(Executor *e, int slot) {
    Slot &sl = e->state[size_t(slot)];
    if (!sl.active || sl.stage < 0) return 1;
    while (sl.scan < sl.first + sl.count && e->lanes[sl.lane].is_done(sl.scan)) ++sl.scan;
    if (sl.scan < sl.first + sl.count) return 0;
    std::atomic_thread_fence(std::memory_order_acquire);
    if (e->err_host[slot]) {
        sl.active = false;
        return -1;
    }
    if (sl.emulated && sl.stage == sl.decide_stage) {
        const int nmod = static_cast<volatile oz::Decision *>(e->dec_host)[slot].nmod;

        sl.moduli = nmod > 0 ? nmod : 0;
        if (nmod <= 0) {  // the native fallback, chosen on the device
            sl.stages.resize(size_t(sl.decide_stage + 1));
            for (const Stage &st : sl.fallback) sl.stages.push_back(st);
            sl.path = 4;
        }
    }
    if (size_t(sl.stage + 1) >= sl.stages.size()) {
        sl.active = false;
        return 1;
    }
    if (e->publish_stage(slot, sl.stage + 1) != BLASX_OK) {
        sl.active = false;
        return -2;
    }
    return 0;
}

void path_of(Executor *e, int slot, int *path, int *moduli) {
    *path = e->state[size_t(slot)].path;
    *moduli = e->state[size_t(slot)].moduli;
}

int pump(Executor *e) { return e->pump_kernel(); }

bool idle(Executor *e) { return !e->pending(); }

int stop(Executor *e) {
    *e->stop_flag = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    if (e->launched) {
        cudaEventSynchronize(e->ev_end);
        e->launched = false;
    }
    *e->stop_flag = 0;
    e->stopping = false;
    e->idle_since = -1.0;
    return BLASX_OK;
}

void counters(Executor *e, long long *launches, long long *tasks) {
    *launches = e->launches;
    unsigned long long n = 0;
    cudaMemcpy(&n, e->tasks_run, sizeof n, cudaMemcpyDeviceToHost);
    *tasks = static_cast<long long>(n);
}

}  // namespace exec
}  // namespace bx
