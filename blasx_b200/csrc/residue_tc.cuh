// residue_tc.cuh -- the INT8 residue GEMM pipeline on the sm_100a tensor
// cores (tcgen05), as device code shared by the standalone kernel
// (ozaki_gemm_tc.cu) and the serving executor (executor.cu).
//
// For every modulus l chosen on the device:
//     U_l[j][i] = (sum_k X_l[j][k] * Y_l[i][k]) mod m_l
// with X_l, Y_l int8 K-major slices and exact INT32 accumulation in TMEM.
// X holds the columns of op(B) (MMA M = 128 rows), Y the rows of op(A)
// (MMA N = 256), so a TMEM lane is a column j of C and a thread of the
// epilogue writes 256 consecutive rows i -- the column-major layout of C.
//
// Warp-specialised pipeline of one CTA:
//   warp 0      TMA producer: 3-D tensor maps (k, row, modulus), 128-byte
//               swizzle, a 4-stage ring of 16 KB (X) + 32 KB (Y) stages;
//   warp 1      holds 512 TMEM columns and issues the MMAs from one thread:
//               4 x tcgen05.mma.kind::i8 (M128 N256 K32) per stage,
//               tcgen05.commit frees the stage; two 256-column accumulators
//               let the epilogue of one tile overlap the MMAs of the next;
//   warps 2..5  epilogue: tcgen05.ld 32x32b.x32, INT32 -> residue mod m_l,
//               16-byte stores of uint8.
// Every mbarrier wait is bounded (a limit in clock cycles, about one second
// by default); on expiry the CTA raises a device error word and an abort flag
// in shared memory, the producer waits (bounded) for its copies in flight,
// the MMA thread waits for its MMAs, and the roles return -- the pipeline
// never spins forever. Everything here has internal linkage: each including
// translation unit holds its own moduli table (upload_moduli).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "ozaki.h"

namespace bx {
namespace oz {
namespace {

constexpr int kStages = 4;
constexpr int kXBytes = kTileJ * kTileK;  // 16 KB
constexpr int kYBytes = kTileI * kTileK;  // 32 KB
constexpr int kStageBytes = kXBytes + kYBytes;
constexpr int kThreadsTC = 192;
constexpr uint32_t kTmemCols = 512;
constexpr int kAccCols = 256;
constexpr long long kWaitCycles = 2000000000LL;  // default wait limit: ~1 s at 1.9 GHz

static __constant__ int c_mod[kMaxModuli];

struct TcArgs {
    int64_t Jp, Ip, Kp;
    uint8_t *U;
    const Decision *dec;
    int *err;
    int tj0, tjn;  // range of j-tiles (128 columns of C each) this launch covers
    int uplo;      // triangular output: 0 all, 1 row - col <= diag, 2 row - col >= diag
    int jtiles;    // j-tiles per column block of X (complex X stacks two blocks)
    int64_t diag;
    long long wait_cycles;  // limit of every mbarrier wait (clock cycles)
    int stall_cta;          // test hook: this CTA skips the loads of its second stage (-1: none)
};

__device__ __forceinline__ uint32_t su32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of `parity` to complete. Returns false when
// `limit` clock cycles have passed or (if given) the CTA abort flag is raised.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag, long long limit) {
    const long long t0 = clock64();
    for (uint32_t it = 0;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63) == 63) {
            if (abort_flag && *abort_flag) return false;
            if (clock64() - t0 > limit) return false;
        }
    }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Shared-memory matrix descriptor: K-major operand, rows of 128 bytes with
// the 128-byte swizzle, 8-row core groups 1024 bytes apart (SBO), sm_100
// descriptor version 1, layout SWIZZLE_128B (2).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = uint64_t((saddr & 0x3FFFF) >> 4);
    // leading byte offset (bits 16..29) stays 0: ignored for swizzled K-major
    d |= uint64_t(1024 >> 4) << 32;    // stride byte offset
    d |= uint64_t(1) << 46;            // descriptor version
    d |= uint64_t(2) << 61;            // SWIZZLE_128B
    return d;
}

// Instruction descriptor, kind::i8: D s32, A s8, B s8, both K-major, N, M.
constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// x mod m in [0, m) for |x| < 2^31, m <= 256: a float quotient estimate is off
// by at most one (|x| * 2^-24 / m < 1), corrected by two compares.
__device__ __forceinline__ uint32_t mod_small(int32_t x, int32_t m, float inv_m) {
    const int32_t q = __float2int_rd(__int2float_rn(x) * inv_m);
    int32_t r = x - q * m;
    r += (r < 0) ? m : 0;
    r -= (r >= m) ? m : 0;
    return uint32_t(r);
}

struct TileCoord {
    int l, tj, ti;
};
__device__ __forceinline__ TileCoord decode(int64_t tile, int tiles_j, int tiles_i, int tj0) {
    constexpr int GJ = 16;  // j-tiles per raster group (operand panels stay in L2)
    const int64_t per_mod = int64_t(tiles_j) * tiles_i;
    TileCoord c;
    c.l = int(tile / per_mod);
    const int64_t t = tile % per_mod;
    const int64_t per_group = int64_t(GJ) * tiles_i;
    const int group = int(t / per_group);
    const int first = group * GJ;
    const int gsize = min(GJ, tiles_j - first);
    const int64_t in = t % per_group;
    c.tj = tj0 + first + int(in % gsize);
    c.ti = int(in / gsize);
    return c;
}

// Triangular output: whether the C tile (rows ti*256.., columns tj*128..) has
// an entry inside the triangle. Every role of the kernel skips the same tiles.
__device__ __forceinline__ bool tile_needed(const TileCoord &c, const TcArgs &a) {
    if (a.uplo == 0) return true;
    const int64_t r0 = int64_t(c.ti) * kTileI, c0 = int64_t(c.tj % a.jtiles) * kTileJ;
    if (a.uplo == 1) return r0 - (c0 + kTileJ - 1) <= a.diag;
    return (r0 + kTileI - 1) - c0 >= a.diag;
}

// Shared-memory layout of one CTA's pipeline: the 4-stage operand ring
// (1024-byte aligned, for the 128-byte swizzle) followed by its mbarriers,
// the TMEM address slot and the CTA abort flag.
constexpr size_t kRingBytes = size_t(kStages) * kStageBytes;
constexpr size_t kPipeBytes = kRingBytes + 128;  // ring + barriers + slot + flag
constexpr size_t kSmemBytes = kPipeBytes + 1024;  // with the alignment slack

struct ResiduePipe {
    uint8_t *ring;
    uint32_t full0, empty0, tfull0, tempty0, done;  // mbarrier addresses
    uint32_t *tmem_slot;
    volatile int *abort_flag;
};

// The pipeline laid out at `base` (1024-byte aligned, kPipeBytes bytes).
__device__ __forceinline__ ResiduePipe residue_pipe_at(uint8_t *base) {
    ResiduePipe p;
    p.ring = base;
    uint64_t *bars = reinterpret_cast<uint64_t *>(base + kRingBytes);
    p.full0 = su32(bars);
    p.empty0 = su32(bars + kStages);
    p.tfull0 = su32(bars + 2 * kStages);
    p.tempty0 = su32(bars + 2 * kStages + 2);
    p.done = su32(bars + 2 * kStages + 4);
    p.tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 5);
    p.abort_flag = reinterpret_cast<volatile int *>(p.tmem_slot + 1);
    return p;
}

// Initialises the barriers and clears the abort flag (one thread; a CTA
// barrier must follow before any role uses them).
__device__ __forceinline__ void residue_pipe_init(const ResiduePipe &p) {
    for (int s = 0; s < kStages; ++s) {
        mbar_init(p.full0 + 8 * s, 1);
        mbar_init(p.empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
        mbar_init(p.tfull0 + 8 * b, 1);
        mbar_init(p.tempty0 + 8 * b, 4);
    }
    mbar_init(p.done, 1);
    *p.abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc_all(uint32_t *slot) {  // one warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free_all(uint32_t tmem) {  // the allocating warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Position of a role thread in the ring and the accumulator pair; it carries
// over from one tile sequence to the next on the same pipeline.
struct RolePos {
    int stage = 0;
    uint32_t phase = 0;
    int acc = 0;
    uint32_t acc_phase = 0;
    uint32_t done_phase = 0;
};

// A sequence of output tiles for one pipeline: either a strided walk over the
// raster order of a launch (first, first + step, ... < end, decoded), or the
// moduli 0 .. nmod-1 of one C tile (tj, ti).
struct TileSeq {
    bool raster;
    int64_t first, step, end;   // raster walk
    int tiles_j, tiles_i, tj0;  // raster geometry
    int tj, ti;                 // one C tile
};
__device__ __forceinline__ TileCoord seq_tile(const TileSeq &q, int64_t s) {
    if (q.raster) return decode(q.first + s * q.step, q.tiles_j, q.tiles_i, q.tj0);
    return TileCoord{int(s), q.tj, q.ti};
}
__device__ __forceinline__ int64_t seq_count(const TileSeq &q, int nmod) {
    if (q.raster) return q.end > q.first ? (q.end - q.first + q.step - 1) / q.step : 0;
    return nmod;
}

// The three roles of the pipeline over the tiles of q, for the calling thread
// (warp 0 lane 0: TMA producer; warp 1 lane 0: MMA issuer; warps 2..5:
// epilogue; every other thread returns at once). On a wait that runs out the
// CTA's abort flag and the device error word are raised, the producer waits
// (bounded) for its copies in flight and the MMA issuer for its MMAs; the
// pipeline must then be initialised again before further use. mapX / mapY:
// generic addresses of the tensor maps (kernel parameters or global memory).
__device__ __forceinline__ void residue_roles(const CUtensorMap *mapX, const CUtensorMap *mapY,
                                              const TcArgs &a, const TileSeq &q, int64_t count,
                                              const ResiduePipe &p, uint32_t tmem, RolePos &pos,
                                              int warp, int lane, bool stall) {
    const int num_kb = int(a.Kp / kTileK);
    volatile int *abort_flag = p.abort_flag;
    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            uint32_t issued = 0, par = 0;  // bit s: stage s has a load issued / its parity
            bool ok = true;
            // test hook: a stalled pipeline issues nothing for its second stage,
            // so that the MMA issuer's wait for that stage runs out
            int skip = stall ? 1 : -1;
            for (int64_t t = 0; t < count && ok; ++t) {
                const TileCoord c = seq_tile(q, t);
                if (!tile_needed(c, a)) continue;
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(p.empty0 + 8 * pos.stage, pos.phase ^ 1, abort_flag, a.wait_cycles)) {
                        ok = false;
                        break;
                    }
                    const bool skip_this = skip == 0;
                    if (skip >= 0) --skip;
                    if (skip_this) {
                        issued &= ~(1u << pos.stage);  // no copy in flight for this stage
                    } else {
                        const uint32_t fb = p.full0 + 8 * pos.stage;
                        mbar_expect_tx(fb, kStageBytes);
                        const uint32_t sx = su32(p.ring + pos.stage * kStageBytes);
                        tma_load_3d(sx, mapX, fb, kb * kTileK, c.tj * kTileJ, c.l);
                        tma_load_3d(sx + kXBytes, mapY, fb, kb * kTileK, c.ti * kTileI, c.l);
                        issued |= 1u << pos.stage;
                        par = (par & ~(1u << pos.stage)) | (pos.phase << pos.stage);
                    }
                    if (++pos.stage == kStages) { pos.stage = 0; pos.phase ^= 1; }
                }
            }
            if (!ok) {
                atomicOr(a.err, 1);
                *abort_flag = 1;
                // wait (bounded) for this thread's copies still in flight
                for (int s = 0; s < kStages; ++s)
                    if (issued & (1u << s)) mbar_wait(p.full0 + 8 * s, (par >> s) & 1u, nullptr, a.wait_cycles);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            constexpr uint32_t idesc = idesc_i8(kTileJ, kTileI);
            bool ok = true;
            for (int64_t t = 0; t < count && ok; ++t) {
                if (!tile_needed(seq_tile(q, t), a)) continue;
                if (!mbar_wait(p.tempty0 + 8 * pos.acc, pos.acc_phase ^ 1, abort_flag, a.wait_cycles)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + uint32_t(pos.acc * kAccCols);
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(p.full0 + 8 * pos.stage, pos.phase, abort_flag, a.wait_cycles)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sx = su32(p.ring + pos.stage * kStageBytes);
                    const uint64_t xd = sdesc(sx), yd = sdesc(sx + kXBytes);
#pragma unroll
                    for (int k = 0; k < kTileK / 32; ++k)
                        umma_i8(d, xd + uint64_t(2 * k), yd + uint64_t(2 * k), idesc, (kb | k) != 0 ? 1u : 0u);
                    umma_commit(p.empty0 + 8 * pos.stage);
                    if (++pos.stage == kStages) { pos.stage = 0; pos.phase ^= 1; }
                }
                if (!ok) break;
                umma_commit(p.tfull0 + 8 * pos.acc);
                if (++pos.acc == 2) { pos.acc = 0; pos.acc_phase ^= 1; }
            }
            if (!ok) {
                atomicOr(a.err, 2);
                *abort_flag = 1;
            }
            // all MMAs of this thread complete before the pipeline is left
            umma_commit(p.done);
            mbar_wait(p.done, pos.done_phase, nullptr, a.wait_cycles);
            pos.done_phase ^= 1;
        }
    } else if (warp < 6) {
        // ---------------- epilogue (warps 2..5) ----------------
        const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
        for (int64_t t = 0; t < count; ++t) {
            const TileCoord c = seq_tile(q, t);
            if (!tile_needed(c, a)) continue;
            const int32_t m = c_mod[c.l];
            const float inv_m = 1.0f / float(m);
            if (!mbar_wait(p.tfull0 + 8 * pos.acc, pos.acc_phase, abort_flag, a.wait_cycles)) {
                if (lane == 0) atomicOr(a.err, 4);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            const int64_t j = int64_t(c.tj) * kTileJ + quarter * 32 + lane;
            uint8_t *out = a.U + int64_t(c.l) * a.Jp * a.Ip + j * a.Ip + int64_t(c.ti) * kTileI;
            const uint32_t tbase = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(pos.acc * kAccCols);
#pragma unroll 1
            for (int ch = 0; ch < kTileI / 32; ++ch) {
                uint32_t r[32];
                tmem_ld32(tbase + uint32_t(ch * 32), r);
                uint32_t w[8];
#pragma unroll
                for (int qq = 0; qq < 8; ++qq) {
                    w[qq] = mod_small(int32_t(r[4 * qq]), m, inv_m) |
                            (mod_small(int32_t(r[4 * qq + 1]), m, inv_m) << 8) |
                            (mod_small(int32_t(r[4 * qq + 2]), m, inv_m) << 16) |
                            (mod_small(int32_t(r[4 * qq + 3]), m, inv_m) << 24);
                }
                uint4 *o = reinterpret_cast<uint4 *>(out + ch * 32);
                o[0] = make_uint4(w[0], w[1], w[2], w[3]);
                o[1] = make_uint4(w[4], w[5], w[6], w[7]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(p.tempty0 + 8 * pos.acc);
            if (++pos.acc == 2) { pos.acc = 0; pos.acc_phase ^= 1; }
        }
    }
}

// ---- tensor maps (host) ------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// 3-D map over [kMaxModuli][rows][Kp] int8 with a (128 k, box_rows, 1) box.
int make_map(CUtensorMap *map, const void *base, int64_t rows, int64_t kp, int box_rows) {
    auto enc = encode_fn();
    if (!enc) return set_error(BLASX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {cuuint64_t(kp), cuuint64_t(rows), cuuint64_t(kMaxModuli)};
    cuuint64_t strides[2] = {cuuint64_t(kp), cuuint64_t(rows * kp)};
    cuuint32_t box[3] = {cuuint32_t(kTileK), cuuint32_t(box_rows), 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(base), dims, strides,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(BLASX_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
    return BLASX_OK;
}

// Uploads the moduli to this translation unit's constant memory on the
// current device.
inline cudaError_t upload_moduli() { return cudaMemcpyToSymbol(c_mod, kModuli, sizeof(kModuli)); }

}  // namespace
}  // namespace oz
}  // namespace bx
