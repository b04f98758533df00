// tile_plan.h -- host-side tile schedule and HBM tile-cache simulation.
//
// Replaces the reference's task queue (blas/blasx_task_queue.c), its
// per-GPU LRU tile cache indexed by a red-black tree keyed on host addresses
// (blas/LRU.c, blas/red_black_tree.c, blas/blasx_mem_control.c:222-340) and
// its reader refcounts (blas/blasx_mem_control.c:45-63) with one planner:
//   * C is cut into T x T tiles (edge tiles clipped, as margin_adjustment in
//     blas/blasx_mem_control.c:24-42) visited in bands of two tile rows,
//     column by column inside a band, snaking, so the tiles of A and B in
//     use are reused by the next C tiles (the plain row-by-row snake when
//     bands would load more tiles);
//   * every K-step of a C tile needs one A tile and one B tile; they live in
//     fixed-size slots of an HBM arena whose size is an explicit byte budget
//     (the reference has none: it evicts when cudaMalloc fails);
//   * the tile index is a hash map keyed on (operand, tile row, tile column);
//   * eviction is Belady's (evict the resident tile whose next use is
//     farthest away -- the schedule is known up front) or LRU (the
//     reference's policy), never a tile pinned by the current K-step.
// The planner is pure host code: it decides, the executor (tile_engine.cu)
// turns each step into stream-ordered copies, kernels and events.
#pragma once

#include <cstdint>
#include <vector>

namespace bx {

struct TileKey {
    int op;  // 0 = A, 1 = B
    int r, c;
    bool operator==(const TileKey &o) const { return op == o.op && r == o.r && c == o.c; }
};

// One operand use of one K-step.
struct TileUse {
    TileKey key;
    int slot;      // arena slot holding the tile
    bool load;     // miss: copy the tile host -> device into `slot`
    int evicted;   // 1 when `slot` held another tile that was dropped
};

// One K-step of one C tile: C(i, j) (+)= op(A)(i, k) op(B)(k, j).
struct TileStep {
    int i, j, k;
    bool first_k, last_k;  // first / last K-step of this C tile
    TileUse a, b;
};

struct TilePlan {
    int tiles_m = 0, tiles_n = 0, tiles_k = 0;
    int slots = 0;
    std::vector<TileStep> steps;
    int64_t loads = 0, hits = 0, evictions = 0;
};

enum TilePolicy { kBelady = 0, kLru = 1 };

// Slots of the arena reserved for C tiles (compute / write-back overlap).
constexpr int kCTileSlots = 3;

// Plans an (M x N x K) GEMM with tile edge T and `slots` operand slots
// (slots >= 2). Returns false when slots < 2.
bool plan_tiles(int64_t M, int64_t N, int64_t K, int64_t T, int slots, int policy, TilePlan *out);

}  // namespace bx
