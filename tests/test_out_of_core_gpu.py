"""GPU tests of the out-of-core path: a small HBM budget forces the tile
cache with evictions; results are checked against the oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture
def small_cache(blx):
    blx.set_hbm_budget(64 << 20)
    blx.set_tile(512)
    prev = blx.set_dgemm_mode(blx.MODE_NATIVE)
    yield blx
    blx.set_hbm_budget(0)
    blx.set_tile(0)
    blx.set_dgemm_mode(prev)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_out_of_core_dgemm(small_cache, ta, tb):
    blx = small_cache
    M, N, K = 3001, 2500, 2047
    ra, ca = oracle.shape_of_op(ta, M, K)
    rb, cb = oracle.shape_of_op(tb, K, N)
    A = oracle.uniform((ra + 1, ca), np.float64, 3)
    B = oracle.uniform((rb, cb), np.float64, 4)
    C0 = oracle.uniform((M + 3, N), np.float64, 5)
    C = C0.copy(order="F")
    blx.cblas_dgemm(102, oracle.TRANS_OF[ta], oracle.TRANS_OF[tb], M, N, K, 1.5, A, ra + 1, B, rb, -0.25, C, M + 3)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    st = blx.call_stats()
    assert st["tile"] == 512 and st["evictions"] > 0 and st["cache_misses"] > 0
    rng = np.random.default_rng(1)
    ii = rng.integers(0, M, 3000); jj = rng.integers(0, N, 3000)
    val, bound = oracle.dd_entries(ta, tb, M, N, K, 1.5, A, ra + 1, B, rb, -0.25, C0, M + 3, ii, jj)
    ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float64)
    assert ratio <= 1.0
    np.testing.assert_array_equal(C[M:, :], C0[M:, :])


def test_out_of_core_zgemm_and_beta_zero(small_cache):
    blx = small_cache
    M, N, K = 1500, 1300, 1100
    A = oracle.uniform((K, M), np.complex128, 7)
    B = oracle.uniform((N, K), np.complex128, 8)
    C = np.full((M, N), np.nan, dtype=np.complex128, order="F")  # beta = 0: C never read
    blx.cblas_zgemm(102, 113, 113, M, N, K, 1 - 0.5j, A, K, B, N, 0, C, M)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    assert blx.call_stats()["evictions"] > 0
    want = (1 - 0.5j) * (A.conj().T @ B.conj().T)
    np.testing.assert_allclose(C, want, rtol=1e-12, atol=1e-11)


@pytest.fixture
def small_cache_emulated(blx):
    blx.set_hbm_budget(64 << 20)
    blx.set_tile(512)
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI)
    yield blx
    blx.set_hbm_budget(0)
    blx.set_tile(0)
    blx.set_dgemm_mode(prev)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
def test_out_of_core_dgemm_emulated_steps(small_cache_emulated, ta, tb):
    """Every K-step on the emulated path (scratch carved from the budget)."""
    blx = small_cache_emulated
    M, N, K = 3001, 2500, 2047
    ra, ca = oracle.shape_of_op(ta, M, K)
    rb, cb = oracle.shape_of_op(tb, K, N)
    A = oracle.uniform((ra + 1, ca), np.float64, 13)
    B = oracle.uniform((rb, cb), np.float64, 14)
    C0 = oracle.uniform((M + 3, N), np.float64, 15)
    C = C0.copy(order="F")
    blx.cblas_dgemm(102, oracle.TRANS_OF[ta], oracle.TRANS_OF[tb], M, N, K, 1.5, A, ra + 1, B, rb, -0.25, C, M + 3)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    st = blx.call_stats()
    assert st["path"] == 2 and st["moduli"] > 0
    assert st["tile"] == 512 and st["evictions"] > 0
    rng = np.random.default_rng(2)
    ii = rng.integers(0, M, 3000); jj = rng.integers(0, N, 3000)
    val, bound = oracle.dd_entries(ta, tb, M, N, K, 1.5, A, ra + 1, B, rb, -0.25, C0, M + 3, ii, jj)
    ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float64)
    assert ratio <= 1.0
    np.testing.assert_array_equal(C[M:, :], C0[M:, :])


def test_out_of_core_zgemm_emulated_steps(small_cache_emulated):
    blx = small_cache_emulated
    M, N, K = 1500, 1300, 1100
    A = oracle.uniform((K, M), np.complex128, 17)
    B = oracle.uniform((N, K), np.complex128, 18)
    C = np.full((M, N), np.nan, dtype=np.complex128, order="F")  # beta = 0: C never read
    blx.cblas_zgemm(102, 113, 113, M, N, K, 1 - 0.5j, A, K, B, N, 0, C, M)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    st = blx.call_stats()
    assert st["path"] == 2 and st["evictions"] > 0
    want = (1 - 0.5j) * (A.conj().T @ B.conj().T)
    np.testing.assert_allclose(C, want, rtol=1e-12, atol=1e-11)


def test_out_of_core_auto_falls_back_per_step(blx):
    """Auto mode on a wide exponent spread: the K-steps (2048^3, large enough
    for auto mode to pick the emulated path) each decide on the device to
    run the native kernel; the result is still the FP64 one."""
    blx.set_hbm_budget(600 << 20)
    blx.set_tile(2048)
    prev = blx.set_dgemm_mode(blx.MODE_AUTO)
    try:
        M, N, K = 6144, 6000, 6144  # every K-step 2048 deep
        A = oracle.spread((M, K), 21, 6.0)
        B = oracle.spread((K, N), 22, 6.0)
        C0 = oracle.uniform((M, N), np.float64, 23)
        C = C0.copy(order="F")
        blx.cblas_dgemm(102, 111, 111, M, N, K, 1.0, A, M, B, K, 0.5, C, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        st = blx.call_stats()
        assert st["path"] == 4 and st["moduli"] == 0 and st["evictions"] > 0
        rng = np.random.default_rng(3)
        ii = rng.integers(0, M, 2000); jj = rng.integers(0, N, 2000)
        val, bound = oracle.dd_entries("N", "N", M, N, K, 1.0, A, M, B, K, 0.5, C0, M, ii, jj)
        ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float64)
        assert ratio <= 1.0
    finally:
        blx.set_hbm_budget(0)
        blx.set_tile(0)
        blx.set_dgemm_mode(prev)
