"""GPU tests of the error paths, driven without faulting the GPU.

* A bounded wait of the INT8 residue GEMM runs out: a test hook makes CTA 0
  issue no loads for one pipeline stage and limits every wait to about one
  millisecond. The kernel raises its device error word, drains its copies
  and MMAs, frees its tensor memory and returns; the host call reports
  BLASX_ERR_TIMEOUT, and the next call (hook disarmed) is correct -- so the
  context stayed usable and no tensor memory leaked.
* The same in the serving loop: the stalled request fails alone, the loop
  keeps serving.
* A device allocation fails (test hook, nothing is allocated): every host
  pipeline returns BLASX_ERR_NOMEM with C (or B) untouched, drains its streams
  before freeing what it had, and the next call is correct.

The reference has no error path to compare with: it assert()s on every CUDA
failure (blas/LRU.c:118,134).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

WAIT = 2_000_000  # clock cycles, about 1 ms


def sampled(C, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, ldc, dt, n=1000, seed=0):
    rng = np.random.default_rng(seed)
    ii = rng.integers(0, M, n); jj = rng.integers(0, N, n)
    val, bound = oracle.dd_entries(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, ldc, ii, jj)
    return oracle.componentwise_ratio(C, ii, jj, val, bound, K, dt)[0]


@pytest.fixture
def mode(blx):
    prev = blx.set_dgemm_mode(blx.MODE_AUTO)
    yield blx
    blx.set_dgemm_mode(prev)
    blx.test_stall_residue_gemm(0, 1)
    blx.test_fail_allocation(0)


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_residue_gemm_wait_runs_out(mode, dt):
    blx = mode
    blx.set_dgemm_mode(blx.MODE_OZAKI)
    M, N, K = 1024, 768, 1024
    A = oracle.uniform((M, K), dt, 1)
    B = oracle.uniform((K, N), dt, 2)
    C0 = oracle.uniform((M, N), dt, 3)
    fn = blx.cblas_dgemm if dt == np.float64 else blx.cblas_zgemm
    alpha, beta = (1.5, 0.5) if dt == np.float64 else (1.5 - 0.5j, 0.5 + 0.25j)
    for _ in range(2):  # twice: the first recovery leaves the context as it was
        assert blx.test_stall_residue_gemm(1, WAIT) == blx.BLASX_OK
        C = C0.copy(order="F")
        fn(102, 111, 111, M, N, K, alpha, A, M, B, K, beta, C, M)
        assert blx.last_status() == blx.BLASX_ERR_TIMEOUT, blx.last_error()
        assert "wait" in blx.last_error()
        C = C0.copy(order="F")
        fn(102, 111, 111, M, N, K, alpha, A, M, B, K, beta, C, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert blx.call_stats()["path"] == 2
        assert sampled(C, "N", "N", M, N, K, alpha, A, M, B, K, beta, C0, M, dt) <= 1.0


def test_serving_request_timeout_fails_alone(mode):
    blx = mode
    M = N = 2048
    K = 1536  # emulated in auto mode
    A = oracle.uniform((M, K), np.float64, 11)
    B = oracle.uniform((K, N), np.float64, 12)
    C0 = oracle.uniform((M, N), np.float64, 13)
    blx.serve_start(0, 0, 4)
    try:
        blx.test_stall_residue_gemm(1, WAIT)
        C = C0.copy(order="F")
        blx.cblas_dgemm(102, 111, 111, M, N, K, 1.0, A, M, B, K, 0.5, C, M)
        assert blx.last_status() == blx.BLASX_ERR_TIMEOUT, blx.last_error()
        st = blx.serve_stats()
        assert st["failed"] == 1
        C = C0.copy(order="F")
        blx.cblas_dgemm(102, 111, 111, M, N, K, 1.0, A, M, B, K, 0.5, C, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert sampled(C, "N", "N", M, N, K, 1.0, A, M, B, K, 0.5, C0, M, np.float64) <= 1.0
        st = blx.serve_stats()
        assert st["failed"] == 1 and st["completed"] == 2
    finally:
        blx.serve_stop()


def _gemm_case(blx, dt, M, N, K, budget):
    A = oracle.uniform((M, K), dt, 21)
    B = oracle.uniform((K, N), dt, 22)
    C0 = oracle.uniform((M, N), dt, 23)
    fn = {np.float64: blx.cblas_dgemm, np.complex128: blx.cblas_zgemm, np.float32: blx.cblas_sgemm}[dt]
    alpha, beta = (1.5, -0.25) if dt != np.complex128 else (1.5 + 0.5j, -0.25)

    def call():
        C = C0.copy(order="F")
        fn(102, 111, 111, M, N, K, alpha, A, M, B, K, beta, C, M)
        return C

    def check(C):
        return sampled(C, "N", "N", M, N, K, alpha, A, M, B, K, beta, C0, M, dt) <= 1.0

    return call, check, C0


@pytest.mark.parametrize("case", ["native", "emulated", "emulated_kblocks", "out_of_core"])
def test_allocation_failure_returns_nomem(mode, case):
    blx = mode
    budget = 0
    if case == "native":
        blx.set_dgemm_mode(blx.MODE_NATIVE)
        M, N, K = 900, 700, 500
    elif case == "emulated":
        blx.set_dgemm_mode(blx.MODE_OZAKI)
        M, N, K = 900, 700, 500
    elif case == "emulated_kblocks":
        blx.set_dgemm_mode(blx.MODE_OZAKI)
        M, N, K = 700, 600, 4608  # two K-blocks
    else:
        blx.set_dgemm_mode(blx.MODE_NATIVE)
        M, N, K = 2048, 2048, 2048
        budget = 48 << 20  # the operands do not fit: tile cache of 512^2 tiles
    blx.set_hbm_budget(budget)
    if case == "out_of_core":
        blx.set_tile(512)
    try:
        if case == "out_of_core":
            blx.finalize()  # the tile arena is allocated again by the next call
        call, check, C0 = _gemm_case(blx, np.float64, M, N, K, budget)
        failures = 0
        for nth in range(1, 8):
            blx.test_fail_allocation(nth)
            C = call()
            st = blx.last_status()
            blx.test_fail_allocation(0)
            if st == blx.BLASX_ERR_NOMEM:
                failures += 1
                # every allocation comes before the first copy back: C is untouched
                assert np.array_equal(C, C0)
            else:
                assert st == blx.BLASX_OK, blx.last_error()
                assert check(C)
            if case == "out_of_core":
                blx.finalize()
        assert failures >= 1
        C = call()
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert check(C)
    finally:
        blx.set_hbm_budget(0)
        blx.set_tile(0)


def test_allocation_failure_in_trsm(mode):
    blx = mode
    n, nrhs = 1500, 700
    rng = np.random.default_rng(5)
    A = np.asfortranarray(np.tril(rng.uniform(-1, 1, (n, n))) + n * np.eye(n))
    B0 = oracle.uniform((n, nrhs), np.float64, 31)
    failures = 0
    for nth in range(1, 8):
        blx.test_fail_allocation(nth)
        B = B0.copy(order="F")
        blx.cblas_dtrsm(102, 141, 122, 111, 131, n, nrhs, 2.0, A, n, B, n)
        st = blx.last_status()
        blx.test_fail_allocation(0)
        if st == blx.BLASX_ERR_NOMEM:
            failures += 1
            assert np.array_equal(B, B0)
        else:
            assert st == blx.BLASX_OK, blx.last_error()
    assert failures >= 1
    B = B0.copy(order="F")
    blx.cblas_dtrsm(102, 141, 122, 111, 131, n, nrhs, 2.0, A, n, B, n)
    assert blx.last_status() == blx.BLASX_OK
    np.testing.assert_allclose(A @ B, 2.0 * B0, rtol=1e-10, atol=1e-10)
