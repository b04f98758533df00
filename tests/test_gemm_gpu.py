"""GPU parity tests: the CUDA path against the reference's own outputs
(tests/golden) and the double-double oracle, through the C ABI."""
import threading

import numpy as np
import pytest

import oracle
from golden_cases import cases, edge_cases, tol_ratio

pytestmark = pytest.mark.gpu

ORDER_COL = 102


def run_case(blx, c, C=None, mode=None):
    C = c["C0"].copy(order="F") if C is None else C
    fn = {np.float64: blx.cblas_dgemm, np.float32: blx.cblas_sgemm, np.complex128: blx.cblas_zgemm,
          np.complex64: blx.cblas_cgemm}[c["dt"]]
    fn(ORDER_COL, oracle.TRANS_OF[c["ta"]], oracle.TRANS_OF[c["tb"]], c["M"], c["N"], c["K"], c["alpha"],
       c["A"], c["lda"], c["B"], c["ldb"], c["beta"], C, c["ldc"])
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    return C


@pytest.mark.parametrize("tag", ["d", "s", "z", "c"])
def test_golden_cases(blx, golden, tag):
    for c in cases(golden, tags=(tag,)):
        C = run_case(blx, c)
        r = tol_ratio(c, C)
        assert r <= 1.0, (c["key"], r)
        np.testing.assert_array_equal(C[c["M"]:, :], c["C0"][c["M"]:, :])


def test_golden_edge_cases(blx, golden):
    for c in edge_cases(golden):
        C = c["C0"].copy(order="F")
        blx.cblas_dgemm(ORDER_COL, 111, 111, c["M"], c["N"], c["K"], c["alpha"], c["A"], c["lda"], c["B"],
                        c["ldb"], c["beta"], C, c["ldc"])
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert np.all(np.isfinite(C)), c["key"]
        np.testing.assert_allclose(C, c["C"], rtol=1e-15, atol=1e-15)


def test_f77_wrappers(blx, golden):
    for c in list(cases(golden, tags=("d", "s", "z", "c")))[::7]:
        C = c["C0"].copy(order="F")
        fn = {np.float64: blx.dgemm_, np.float32: blx.sgemm_, np.complex128: blx.zgemm_,
              np.complex64: blx.cgemm_}[c["dt"]]
        fn(c["ta"].lower(), c["tb"], c["M"], c["N"], c["K"], c["alpha"], c["A"], c["lda"], c["B"], c["ldb"],
           c["beta"], C, c["ldc"])
        assert tol_ratio(c, C) <= 1.0, c["key"]


@pytest.mark.parametrize("dt", [np.float64, np.float32, np.complex128, np.complex64])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T"), ("C", "N"), ("N", "C"), ("C", "C")])
def test_random_vs_dd_oracle(blx, dt, ta, tb):
    cplx = dt in (np.complex128, np.complex64)
    if not cplx and "C" in (ta, tb):
        pytest.skip("ConjTrans on real data is Trans (covered)")
    rng = np.random.default_rng(7)
    M, N, K = 517, 263, 1031
    ra, ca = oracle.shape_of_op(ta, M, K)
    rb, cb = oracle.shape_of_op(tb, K, N)
    A = oracle.uniform((ra + 3, ca), dt, 11)
    B = oracle.uniform((rb + 1, cb), dt, 12)
    C0 = oracle.uniform((M + 2, N), dt, 13)
    alpha, beta = (1.5, -0.25) if not cplx else (1.5 - 0.5j, -0.25 + 0.75j)
    C = C0.copy(order="F")
    fn = {np.float64: blx.cblas_dgemm, np.float32: blx.cblas_sgemm, np.complex128: blx.cblas_zgemm,
          np.complex64: blx.cblas_cgemm}[dt]
    fn(ORDER_COL, oracle.TRANS_OF[ta], oracle.TRANS_OF[tb], M, N, K, alpha, A, ra + 3, B, rb + 1, beta, C, M + 2)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    ii = rng.integers(0, M, 2000); jj = rng.integers(0, N, 2000)
    val, bound = oracle.dd_entries(ta, tb, M, N, K, alpha, A, ra + 3, B, rb + 1, beta, C0, M + 2, ii, jj)
    ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, dt)
    assert ratio <= 1.0
    np.testing.assert_array_equal(C[M:, :], C0[M:, :])


def test_row_major(blx):
    M, N, K = 300, 200, 150
    A = np.ascontiguousarray(oracle.uniform((M, K), np.float64, 1))  # row-major M x K
    B = np.ascontiguousarray(oracle.uniform((K, N), np.float64, 2))
    C = np.ascontiguousarray(oracle.uniform((M, N), np.float64, 3))
    want = 0.5 * A @ B + 2.0 * C
    blx.cblas_dgemm(101, 111, 111, M, N, K, 0.5, A, K, B, N, 2.0, C, N)
    assert blx.last_status() == blx.BLASX_OK
    np.testing.assert_allclose(C, want, rtol=1e-12, atol=1e-12)
    # transposed row-major operands
    At = np.ascontiguousarray(A.T); C2 = np.zeros((M, N))
    blx.cblas_dgemm(101, 112, 111, M, N, K, 1.0, At, M, B, N, 0.0, C2, N)
    np.testing.assert_allclose(C2, A @ B, rtol=1e-12, atol=1e-12)


def test_device_entry_matches_host(blx):
    torch = pytest.importorskip("torch")
    M, N, K = 640, 384, 512
    A = oracle.uniform((M, K), np.float64, 21); B = oracle.uniform((K, N), np.float64, 22)
    C = oracle.uniform((M, N), np.float64, 23)
    Ch = C.copy(order="F")
    blx.cblas_dgemm(102, 111, 111, M, N, K, 1.25, A, M, B, K, -0.5, Ch, M)
    # torch is column-major-agnostic: pass the transposed (row-major) views' storage
    dA = torch.from_numpy(A.T.copy()).cuda(); dB = torch.from_numpy(B.T.copy()).cuda()
    dC = torch.from_numpy(C.T.copy()).cuda()
    st = blx.gemm_device("N", "N", M, N, K, 1.25, dA, M, dB, K, -0.5, dC, M,
                         stream=torch.cuda.current_stream(), dtype="d")
    assert st == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dC.cpu().numpy().T, Ch)


def test_threads_concurrent_calls(blx):
    M, N, K = 257, 129, 300
    results, errs = {}, []

    def worker(t):
        try:
            A = oracle.uniform((M, K), np.float64, 100 + t); B = oracle.uniform((K, N), np.float64, 200 + t)
            C = np.zeros((M, N), order="F")
            blx.cblas_dgemm(102, 111, 111, M, N, K, 1.0, A, M, B, K, 0.0, C, M)
            results[t] = np.abs(C - A @ B).max()
        except Exception as e:  # pragma: no cover
            errs.append(e)

    th = [threading.Thread(target=worker, args=(t,)) for t in range(8)]
    [x.start() for x in th]
    [x.join() for x in th]
    assert not errs
    assert max(results.values()) < 1e-12


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("beta", [0.0, -0.75])
def test_sgemm_native_wide_tile(blx, ta, tb, beta):
    """FP32 on the native path with at least one wave of 128 x 128 tiles (the
    8 x 8-per-thread kernel): ragged in M, N and K, padded leading dimensions;
    with beta = 0, C holds NaN that must not be read."""
    prev = blx.set_dgemm_mode(blx.MODE_NATIVE)
    try:
        M, N, K = 1701, 1509, 999
        ra, ca = oracle.shape_of_op(ta, M, K)
        rb, cb = oracle.shape_of_op(tb, K, N)
        A = oracle.uniform((ra + 5, ca), np.float32, 21)
        B = oracle.uniform((rb + 3, cb), np.float32, 22)
        C0 = oracle.uniform((M + 2, N), np.float32, 23)
        if beta == 0.0:
            C0[:M] = np.nan
        C = C0.copy(order="F")
        blx.cblas_sgemm(ORDER_COL, oracle.TRANS_OF[ta], oracle.TRANS_OF[tb], M, N, K, 1.25, A, ra + 5, B, rb + 3,
                        beta, C, M + 2)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert blx.call_stats()["path"] == 1
        np.testing.assert_array_equal(C[M:, :], C0[M:, :])
        rng = np.random.default_rng(9)
        ii = rng.integers(0, M, 4000); jj = rng.integers(0, N, 4000)
        ii[:4] = [0, M - 1, 127, 128]; jj[:4] = [0, N - 1, 128, 127]  # tile corners and the ragged edge
        Cr = np.nan_to_num(C0)
        val, bound = oracle.dd_entries(ta, tb, M, N, K, 1.25, A, ra + 5, B, rb + 3, beta, Cr, M + 2, ii, jj)
        ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float32)
        assert ratio <= 1.0
    finally:
        blx.set_dgemm_mode(prev)


def test_ssyrk_native_wide_tile(blx):
    """The triangular mask of the 128 x 128 FP32 kernel: SSYRK upper on the
    native path, the other triangle bit for bit unchanged."""
    prev = blx.set_dgemm_mode(blx.MODE_NATIVE)
    try:
        N, K = 1900, 700
        A = oracle.uniform((N, K), np.float32, 31)
        C0 = oracle.uniform((N, N), np.float32, 32)
        C = C0.copy(order="F")
        blx.cblas_ssyrk(ORDER_COL, 121, 111, N, K, 0.5, A, N, 2.0, C, N)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        m = oracle.tri_mask("U", N)
        np.testing.assert_array_equal(C[~m], C0[~m])
        rng = np.random.default_rng(10)
        ii = rng.integers(0, N, 4000); jj = rng.integers(0, N, 4000)
        keep = ii <= jj
        ii, jj = ii[keep], jj[keep]
        val, bound = oracle.dd_entries("N", "T", N, N, K, 0.5, A, N, A, N, 2.0, C0, N, ii, jj)
        ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float32)
        assert ratio <= 1.0
    finally:
        blx.set_dgemm_mode(prev)
