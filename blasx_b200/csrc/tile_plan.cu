// tile_plan.cu -- tile schedule and HBM tile-cache simulation (see
// tile_plan.h). Host code only; also exported as blasx_tile_plan so the
// schedule can be inspected (and tested) without a GPU.
#include <algorithm>
#include <limits>
#include <set>
#include <unordered_map>

#include "../../include/blasx_b200.h"
#include "tile_plan.h"

namespace bx {

namespace {

struct KeyHash {
    size_t operator()(const TileKey &k) const {
        return (size_t(k.op) * 1000003u + size_t(k.r)) * 1000003u + size_t(k.c);
    }
};

}  // namespace

namespace {

// The reference string: C tiles in `rows`-row bands, the bands taken top to
// bottom, a band's tiles column by column (the columns snaking from band to
// band, the rows inside a column snaking from column to column), K-steps
// inside. rows = 1 is the plain snake order (row by row, alternate rows
// reversed).
void band_order(TilePlan &p, int rows) {
    p.steps.clear();
    for (int b0 = 0, band = 0; b0 < p.tiles_m; b0 += rows, ++band) {
        const int b1 = std::min(p.tiles_m, b0 + rows);
        for (int jj = 0; jj < p.tiles_n; ++jj) {
            const int j = band % 2 == 0 ? jj : p.tiles_n - 1 - jj;
            for (int ii = 0; ii < b1 - b0; ++ii) {
                const int i = jj % 2 == 0 ? b0 + ii : b1 - 1 - ii;
                for (int k = 0; k < p.tiles_k; ++k) {
                    TileStep s;
                    s.i = i; s.j = j; s.k = k;
                    s.first_k = (k == 0);
                    s.last_k = (k == p.tiles_k - 1);
                    s.a = TileUse{TileKey{0, i, k}, -1, false, 0};
                    s.b = TileUse{TileKey{1, k, j}, -1, false, 0};
                    p.steps.push_back(s);
                }
            }
        }
    }
}

// Simulates the cache over p.steps: slot, load and eviction of every use.
void simulate(TilePlan &p, int slots, int policy) {
    p.loads = p.hits = p.evictions = 0;
    const int64_t nuse = int64_t(p.steps.size()) * 2;
    auto use_key = [&](int64_t u) -> const TileKey & {
        return (u & 1) ? p.steps[size_t(u >> 1)].b.key : p.steps[size_t(u >> 1)].a.key;
    };
    // next use of the same tile after every use (for Belady)
    std::vector<int64_t> next(size_t(nuse), std::numeric_limits<int64_t>::max());
    {
        std::unordered_map<TileKey, int64_t, KeyHash> last;
        for (int64_t u = nuse - 1; u >= 0; --u) {
            auto it = last.find(use_key(u));
            if (it != last.end()) next[size_t(u)] = it->second;
            last[use_key(u)] = u;
        }
    }
    std::unordered_map<TileKey, int, KeyHash> where;  // resident tile -> slot
    std::vector<TileKey> holder(size_t(slots), TileKey{-1, -1, -1});
    std::vector<int64_t> prio(size_t(slots), 0);  // Belady: next use; LRU: last use
    std::set<std::pair<int64_t, int>> order;       // (priority, slot) of occupied slots
    std::vector<int> free_slots;
    for (int s = slots - 1; s >= 0; --s) free_slots.push_back(s);

    for (int64_t u = 0; u < nuse; ++u) {
        TileStep &st = p.steps[size_t(u >> 1)];
        TileUse &use = (u & 1) ? st.b : st.a;
        const TileKey &key = use.key;
        // the partner operand of this K-step must stay resident
        const TileKey *pinned = (u & 1) ? &st.a.key : nullptr;
        const int64_t pr = policy == kBelady ? next[size_t(u)] : u;
        auto it = where.find(key);
        if (it != where.end()) {
            const int s = it->second;
            order.erase({prio[size_t(s)], s});
            prio[size_t(s)] = policy == kBelady ? pr : u;
            order.insert({prio[size_t(s)], s});
            use.slot = s;
            use.load = false;
            ++p.hits;
            continue;
        }
        int s;
        if (!free_slots.empty()) {
            s = free_slots.back();
            free_slots.pop_back();
        } else {
            // Belady: largest next use; LRU: smallest last use; skip the pinned tile
            auto pick = order.end();
            if (policy == kBelady) {
                for (auto r = order.rbegin(); r != order.rend(); ++r)
                    if (!(pinned && holder[size_t(r->second)] == *pinned)) {
                        pick = std::prev(r.base());
                        break;
                    }
            } else {
                for (auto f = order.begin(); f != order.end(); ++f)
                    if (!(pinned && holder[size_t(f->second)] == *pinned)) {
                        pick = f;
                        break;
                    }
            }
            s = pick->second;
            order.erase(pick);
            where.erase(holder[size_t(s)]);
            use.evicted = 1;
            ++p.evictions;
        }
        holder[size_t(s)] = key;
        where[key] = s;
        prio[size_t(s)] = pr;
        order.insert({pr, s});
        use.slot = s;
        use.load = true;
        ++p.loads;
    }
}

}  // namespace

bool plan_tiles(int64_t M, int64_t N, int64_t K, int64_t T, int slots, int policy, TilePlan *out) {
    if (slots < 2 || T <= 0 || M <= 0 || N <= 0 || K <= 0) return false;
    TilePlan &p = *out;
    p = TilePlan{};
    p.tiles_m = int((M + T - 1) / T);
    p.tiles_n = int((N + T - 1) / T);
    p.tiles_k = int((K + T - 1) / T);
    p.slots = slots;
    // Bands of two tile rows, unless they load more tiles than the snake
    // order: the snake's first row of C tiles needs every B tile, and while
    // those cross the host link the compute waits; a band needs them for
    // twice the C tiles, so the link keeps pace with the compute sooner.
    band_order(p, 1);
    simulate(p, slots, policy);
    if (p.tiles_m >= 2) {
        TilePlan b = p;
        band_order(b, 2);
        simulate(b, slots, policy);
        if (b.loads <= p.loads) p = std::move(b);
    }
    return true;
}

}  // namespace bx

extern "C" int blasx_tile_plan(long long M, long long N, long long K, long long tile,
                               long long budget_bytes, int elem_bytes, int policy,
                               blasx_tile_plan_stats *out) {
    if (!out || elem_bytes <= 0 || tile <= 0) return BLASX_ERR_ARG;
    const long long slot_bytes = tile * tile * elem_bytes;
    const long long slots = budget_bytes / slot_bytes - bx::kCTileSlots;
    bx::TilePlan p;
    if (slots < 2 || slots > (1 << 30) || !bx::plan_tiles(M, N, K, tile, int(slots), policy, &p))
        return BLASX_ERR_ARG;
    out->tiles_m = p.tiles_m;
    out->tiles_n = p.tiles_n;
    out->tiles_k = p.tiles_k;
    out->slots = p.slots;
    out->steps = (long long)p.steps.size();
    out->tile_loads = p.loads;
    out->tile_hits = p.hits;
    out->evictions = p.evictions;
    // H2D bytes of the operand loads (edge tiles clipped)
    double h2d = 0;
    for (const bx::TileStep &s : p.steps) {
        auto ext = [&](long long idx, long long n) { return double(std::min(tile, n - idx * tile)); };
        if (s.a.load) h2d += ext(s.i, M) * ext(s.k, K) * elem_bytes;
        if (s.b.load) h2d += ext(s.k, K) * ext(s.j, N) * elem_bytes;
    }
    out->operand_h2d_bytes = h2d;
    out->min_operand_h2d_bytes = double(elem_bytes) * (double(M) * K + double(K) * N);
    return BLASX_OK;
}
