"""CPU tests of the out-of-core tile planner (HBM tile cache simulation)."""
import pytest

G = 1 << 30


def test_c2_config_reaches_minimum_h2d(blx):
    # 40960^3 FP64 with a 24 GB cache: every operand element crosses PCIe once
    for tile in (1024, 2048, 3072, 4096, 8192):
        for pol in (blx.POLICY_BELADY, blx.POLICY_LRU):
            s = blx.tile_plan(40960, 40960, 40960, tile, 24 * G, 8, pol)
            assert s["operand_h2d_bytes"] == pytest.approx(s["min_operand_h2d_bytes"])
            assert s["tile_loads"] + s["tile_hits"] == 2 * s["steps"]


def test_belady_never_loads_more_than_lru(blx):
    for (m, n, k, budget_tiles) in [(8, 8, 8, 6), (5, 7, 3, 4), (10, 3, 9, 5), (4, 4, 16, 3)]:
        t = 256
        budget = (budget_tiles + 3) * t * t * 8  # + 3 C slots
        b = blx.tile_plan(m * t, n * t, k * t, t, budget, 8, blx.POLICY_BELADY)
        l = blx.tile_plan(m * t, n * t, k * t, t, budget, 8, blx.POLICY_LRU)
        assert b["slots"] == budget_tiles
        assert b["tile_loads"] <= l["tile_loads"]
        # each distinct tile is loaded at least once
        assert b["tile_loads"] >= m * k + k * n


def test_ragged_edges_and_minimum(blx):
    # ragged sizes: edge tiles are clipped; a budget holding everything loads each tile once
    M, N, K, t = 3001, 1777, 999, 512
    s = blx.tile_plan(M, N, K, t, 1 << 40, 8, blx.POLICY_LRU)
    assert (s["tiles_m"], s["tiles_n"], s["tiles_k"]) == (6, 4, 2)
    assert s["evictions"] == 0
    assert s["operand_h2d_bytes"] == pytest.approx(8.0 * (M * K + K * N))


def test_budget_too_small_is_rejected(blx):
    with pytest.raises(ValueError):
        blx.tile_plan(4096, 4096, 4096, 1024, 1024 * 1024 * 8 * 4, 8)  # 4 slots - 3 C slots = 1


# ---- an independent restatement of the planner's visiting order and cache ----

def _order(tm, tn, tk, rows):
    """C tiles in `rows`-row bands, each band column by column (columns
    snaking from band to band, rows inside a column snaking from column to
    column), K-steps inside; rows = 1 is the row-by-row snake."""
    uses = []
    for band, b0 in enumerate(range(0, tm, rows)):
        b1 = min(tm, b0 + rows)
        for jj in range(tn):
            j = jj if band % 2 == 0 else tn - 1 - jj
            for ii in range(b1 - b0):
                i = b0 + ii if jj % 2 == 0 else b1 - 1 - ii
                for k in range(tk):
                    uses += [("A", i, k), ("B", k, j)]
    return uses


def _simulate(uses, slots, belady):
    """Loads and evictions of a cache of `slots` operand tiles over the use
    string. Belady evicts the resident tile used again farthest ahead, LRU the
    least recently used; the other operand of the same K-step is never
    evicted; ties go to the highest slot, free slots are taken lowest first."""
    inf = float("inf")
    nxt = [inf] * len(uses)
    seen = {}
    for u in range(len(uses) - 1, -1, -1):
        nxt[u] = seen.get(uses[u], inf)
        seen[uses[u]] = u
    where, holder, prio = {}, [None] * slots, [0] * slots
    free = list(range(slots - 1, -1, -1))
    loads = evictions = 0
    for u, key in enumerate(uses):
        pr = nxt[u] if belady else u
        if key in where:
            prio[where[key]] = pr
            continue
        if free:
            s = free.pop()
        else:
            pinned = uses[u - 1] if u % 2 else None
            occupied = [(prio[x], x) for x in range(slots) if holder[x] is not None and holder[x] != pinned]
            s = (max(occupied) if belady else min(occupied))[1]
            del where[holder[s]]
            evictions += 1
        holder[s], where[key], prio[s] = key, s, pr
        loads += 1
    return loads, evictions


@pytest.mark.parametrize("tm,tn,tk,slots", [
    (5, 5, 5, 8), (6, 4, 3, 5), (4, 7, 2, 6), (7, 3, 4, 4), (1, 6, 5, 4), (3, 3, 9, 3), (8, 8, 2, 12),
    (3, 2, 2, 5), (3, 2, 2, 8),  # the snake loads fewer (with Belady / with LRU): it is kept
])
@pytest.mark.parametrize("belady", [True, False])
def test_plan_matches_restated_band_and_snake_orders(blx, tm, tn, tk, slots, belady):
    # the planner keeps the two-row bands when they load no more tiles than
    # the row snake; its counts match the restatement exactly
    t = 128
    budget = (slots + 3) * t * t * 8  # + 3 C slots
    pol = blx.POLICY_BELADY if belady else blx.POLICY_LRU
    s = blx.tile_plan(tm * t, tn * t, tk * t, t, budget, 8, pol)
    assert s["slots"] == slots
    snake = _simulate(_order(tm, tn, tk, 1), slots, belady)
    best = snake
    if tm >= 2:
        band = _simulate(_order(tm, tn, tk, 2), slots, belady)
        if band[0] <= snake[0]:
            best = band
    assert (s["tile_loads"], s["evictions"]) == best
    assert s["tile_loads"] + s["tile_hits"] == 2 * s["steps"]
