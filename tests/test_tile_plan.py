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
