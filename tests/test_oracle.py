"""CPU tests: the oracle is pinned against the reference's own outputs."""
import numpy as np
import pytest

import oracle
from golden_cases import cases, edge_cases, tol_ratio


def test_generator_is_stable(golden):
    # the golden inputs are regenerated from seeds; their checksums must match
    for c in cases(golden, tags=("d", "s", "z", "c")):
        np.testing.assert_allclose([np.sum(c["A"]), np.sum(c["B"]), np.sum(c["C0"])], c["sums"], rtol=1e-12, atol=1e-12)


def test_tiled_restatement_matches_reference(golden):
    worst = 0.0
    for c in cases(golden, tags=("d", "s", "z", "c")):
        C = c["C0"].copy(order="F")
        # small block size so the restatement exercises several tiles and ragged edges
        oracle.gemm_tiled(c["ta"], c["tb"], c["M"], c["N"], c["K"], c["alpha"], c["A"], c["lda"],
                          c["B"], c["ldb"], c["beta"], C, c["ldc"], block_dim=16)
        r = tol_ratio(c, C)
        worst = max(worst, r)
        assert r <= 1.0, (c["key"], r)
        # rows beyond M in the ldc padding stay untouched
        np.testing.assert_array_equal(C[c["M"]:, :], c["C0"][c["M"]:, :])


def test_dd_entries_match_reference(golden):
    for c in cases(golden, tags=("d", "s", "z", "c")):
        M, N = c["M"], c["N"]
        ii, jj = np.meshgrid(np.arange(M), np.arange(N), indexing="ij")
        ii, jj = ii.ravel(), jj.ravel()
        val, bound = oracle.dd_entries(c["ta"], c["tb"], M, N, c["K"], c["alpha"], c["A"], c["lda"], c["B"],
                                       c["ldb"], c["beta"], c["C0"], c["ldc"], ii, jj)
        ratio, _ = oracle.componentwise_ratio(c["C"], ii, jj, val, bound, c["K"], c["dt"])
        assert ratio <= 1.0, (c["key"], ratio)


def test_dd_is_more_accurate_than_working_precision():
    # cancellation-heavy dot product: the double-double oracle must get it exactly
    K = 1000
    A = np.zeros((1, K), order="F"); B = np.zeros((K, 1), order="F")
    A[0, 0::2] = 1e16; A[0, 1::2] = -1e16; A[0, 10] += 3.0
    B[:, 0] = 1.0
    val, _ = oracle.dd_entries("N", "N", 1, 1, K, 1.0, A, 1, B, K, 0.0, None, 1, [0], [0])
    assert val[0] == np.sum(A.astype(np.longdouble))


def test_edge_cases_restatement(golden):
    for c in edge_cases(golden):
        C = c["C0"].copy(order="F")
        oracle.gemm_tiled("N", "N", c["M"], c["N"], c["K"], c["alpha"], c["A"], c["lda"], c["B"], c["ldb"],
                          c["beta"], C, c["ldc"])
        np.testing.assert_allclose(C, c["C"], rtol=1e-14, atol=1e-14)
        assert np.all(np.isfinite(C))


def test_openblas_matches_reference(golden):
    try:
        ob = oracle.OpenBLAS()
    except RuntimeError as e:
        pytest.skip(str(e))
    for c in cases(golden, tags=("d", "z", "c")):
        C = c["C0"].copy(order="F")
        ob.gemm(c["ta"], c["tb"], c["M"], c["N"], c["K"], c["alpha"], c["A"], c["lda"], c["B"], c["ldb"],
                c["beta"], C, c["ldc"])
        assert tol_ratio(c, C) <= 1.0, c["key"]


def test_golden_xerbla_lines(golden):
    lines = [str(x) for x in golden["xerbla"]]
    assert any("parameter number 13" in l for l in lines)
    # F77 wrapper: a bad TransB overrides a bad TransA (blas/dgemm.c:140-146)
    xy = [l for l in lines if l.startswith("dgemm_XY")][0]
    assert "parameter number  2" in xy
