"""CPU tests of the SYMM / HEMM / TRMM / TRSM restatement in the oracle and of
the library's argument checking for them, both pinned to the reference: the
fixtures hold the reference's own outputs (its CPU BLAS path, which it uses
for every SYMM / HEMM / TRMM / TRSM call, column-major and row-major) and its
xerbla_ lines (tests/golden/make_golden_symm.py)."""
import os

import numpy as np
import pytest

import oracle
from golden_cases import (rank_k_case, rank_k_check, rank_k_oracle, symm_case, symm_check, symm_keys,
                          symm_oracle)
from test_abi import _capture

GOLDEN_SYMM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "symm_trmm_golden.npz")


@pytest.fixture(scope="session")
def sgolden():
    return np.load(GOLDEN_SYMM)


def test_fixture_counts(sgolden):
    # 4 shapes x 2 sides x 2 triangles column-major, + 4 row-major; per type
    assert len(symm_keys(sgolden, "symm_")) == 4 * 20
    assert len(symm_keys(sgolden, "hemm_")) == 2 * 20
    # 3 shapes x 2 x 2 x trans (2 real, 3 complex) x 2 diags, + one row-major shape
    assert len(symm_keys(sgolden, "trmm_")) == 2 * (48 + 16) + 2 * (72 + 24)
    assert len(symm_keys(sgolden, "trsm_")) == 2 * (48 + 16) + 2 * (72 + 24)


@pytest.mark.parametrize("prefix", ["symm_", "hemm_", "trmm_", "trsm_"])
def test_oracle_matches_reference(sgolden, prefix):
    for key in symm_keys(sgolden, prefix):
        kind, tag, x, al, be, want = symm_case(sgolden, key)
        got = symm_oracle(kind, x, al, be)
        symm_check(kind, x, got, want, al, be)


def test_complete_reads_one_triangle():
    A = np.arange(16, dtype=np.float64).reshape(4, 4, order="F")
    U = oracle.complete("S", "U", A, 4)
    assert np.array_equal(U, np.triu(A) + np.triu(A, 1).T)
    T = oracle.complete("T", "L", A, 4, "U")
    assert np.array_equal(T, np.tril(A, -1) + np.eye(4))
    Z = (A + 1j * A.T).astype(np.complex128)
    H = oracle.complete("H", "L", Z, 4)
    assert np.array_equal(H, H.conj().T) and np.all(np.diag(H).imag == 0)


SYMM_BAD = {1: dict(side=999), 2: dict(uplo=999), 3: dict(M=-1), 4: dict(N=-1), 7: dict(lda=2), 9: dict(ldb=2),
            12: dict(ldc=2)}


@pytest.mark.parametrize("info", sorted(SYMM_BAD))
@pytest.mark.parametrize("fn", ["cblas_dsymm", "cblas_zhemm"])
def test_symm_xerbla_matches_reference(blx, sgolden, fn, info):
    want = [str(l) for l in sgolden["xerbla"] if str(l).startswith(f"{fn}|{info}|")][0].split("|", 2)[2]
    a = dict(side=141, uplo=121, M=4, N=4, lda=4, ldb=4, ldc=4)
    a.update(SYMM_BAD[info])
    dt = np.float64 if fn == "cblas_dsymm" else np.complex128
    A = np.zeros((4, 4), dt); C = np.ones((4, 4), dt, order="F")
    got = _capture(lambda: getattr(blx, fn)(102, a["side"], a["uplo"], a["M"], a["N"], 1.0, A, a["lda"], A,
                                            a["ldb"], 0.0, C, a["ldc"]))
    assert got == want
    assert np.all(C == 1.0) and blx.last_status() == blx.BLASX_ERR_ARG


TRMM_BAD = {1: dict(side=999), 2: dict(uplo=999), 3: dict(trans=999), 4: dict(diag=999), 5: dict(M=-1),
            6: dict(N=-1), 9: dict(lda=2), 11: dict(ldb=2)}


@pytest.mark.parametrize("info", sorted(TRMM_BAD))
@pytest.mark.parametrize("fn", ["cblas_dtrmm", "cblas_dtrsm"])
def test_trmm_xerbla_matches_reference(blx, sgolden, fn, info):
    want = [str(l) for l in sgolden["xerbla"] if str(l).startswith(f"{fn}|{info}|")][0].split("|", 2)[2]
    a = dict(side=141, uplo=121, trans=111, diag=131, M=4, N=4, lda=4, ldb=4)
    a.update(TRMM_BAD[info])
    A = np.zeros((4, 4)); B = np.ones((4, 4), order="F")
    got = _capture(lambda: getattr(blx, fn)(102, a["side"], a["uplo"], a["trans"], a["diag"], a["M"], a["N"], 1.0,
                                            A, a["lda"], B, a["ldb"]))
    assert got == want
    assert np.all(B == 1.0) and blx.last_status() == blx.BLASX_ERR_ARG


@pytest.mark.parametrize("sd,up", [("X", "U"), ("L", "Q"), ("X", "Q")])
@pytest.mark.parametrize("fn", ["dsymm_", "zhemm_"])
def test_f77_symm_errors_match_reference(blx, sgolden, fn, sd, up):
    want = [str(l) for l in sgolden["xerbla"] if str(l).startswith(f"{fn}{sd}{up}|")][0].split("|", 2)[2]
    dt = np.float64 if fn == "dsymm_" else np.complex128
    A = np.zeros((4, 4), dt); C = np.ones((4, 4), dt, order="F")
    got = _capture(lambda: getattr(blx, fn)(sd, up, 4, 4, 1.0, A, 4, A, 4, 0.0, C, 4))
    assert got == want
    assert np.all(C == 1.0)


@pytest.mark.parametrize("chars", ["XUNN", "LQNN", "LUQN", "LUNQ", "XQQQ", "LUQQ"])
@pytest.mark.parametrize("fn", ["dtrmm_", "dtrsm_"])
def test_f77_trmm_errors_match_reference(blx, sgolden, fn, chars):
    want = [str(l) for l in sgolden["xerbla"] if str(l).startswith(f"{fn}{chars}|")][0].split("|", 2)[2]
    A = np.zeros((4, 4)); B = np.ones((4, 4), order="F")
    got = _capture(lambda: getattr(blx, fn)(*chars, 4, 4, 1.0, A, 4, B, 4))
    assert got == want
    assert np.all(B == 1.0)


def test_quick_returns_need_no_gpu(blx):
    C = np.ones((4, 4), order="F")
    blx.cblas_dsymm(102, 141, 121, 0, 4, 1.0, C, 4, C, 4, 0.0, C, 4)
    assert blx.last_status() == blx.BLASX_OK
    blx.cblas_dtrmm(102, 142, 122, 111, 131, 4, 0, 1.0, C, 4, C, 4)
    assert blx.last_status() == blx.BLASX_OK and np.all(C == 1.0)


def test_row_major_uses_the_row_major_leading_dimension(blx):
    """Row-major B and C are M x N with ld >= N (the reference applies the
    column-major rule whatever the Order; its CPU BLAS then rejects such calls)."""
    A = np.zeros((8, 8)); C = np.ones((8, 8), order="F")
    out = _capture(lambda: blx.cblas_dsymm(101, 141, 121, 8, 4, 1.0, A, 8, C, 3, 0.0, C, 8))
    assert "DSYMM  parameter number  9" in out
    out = _capture(lambda: blx.cblas_dtrmm(101, 141, 121, 111, 131, 8, 4, 1.0, A, 8, C, 3))
    assert "DTRMM  parameter number 11" in out and np.all(C == 1.0)
    out = _capture(lambda: blx.cblas_dtrsm(101, 141, 121, 111, 131, 8, 4, 1.0, A, 8, C, 3))
    assert "DTRSM  parameter number 11" in out and np.all(C == 1.0)


RANK_K = ["herk_", "her2k_", "syrk_c", "syr2k_c"]


def rank_k_keys(golden, prefix):
    return [k for k in symm_keys(golden, prefix.split("_")[0] + "_") if k.startswith(prefix)]


def test_rank_k_fixture_counts(sgolden):
    # 4 shapes x 2 triangles x 2 transposes column-major, + 4 row-major; per type
    assert len(rank_k_keys(sgolden, "herk_")) == 2 * 20
    assert len(rank_k_keys(sgolden, "her2k_")) == 2 * 20
    assert len(rank_k_keys(sgolden, "syrk_c")) == 20 and len(rank_k_keys(sgolden, "syr2k_c")) == 20


@pytest.mark.parametrize("prefix", RANK_K)
def test_rank_k_oracle_matches_reference(sgolden, prefix):
    for key in rank_k_keys(sgolden, prefix):
        kind, tag, x, al, be, want = rank_k_case(sgolden, key)
        rank_k_check(x, rank_k_oracle(x, al, be), want, al, be)


HERK_BAD = {1: dict(uplo=999), 2: dict(trans=112), 3: dict(N=-1), 4: dict(K=-1), 7: dict(lda=2), 10: dict(ldc=2)}


@pytest.mark.parametrize("info", sorted(HERK_BAD))
def test_herk_xerbla_matches_reference(blx, sgolden, info):
    want = [str(l) for l in sgolden["xerbla"] if str(l).startswith(f"cblas_zherk|{info}|")][0].split("|", 2)[2]
    a = dict(uplo=121, trans=111, N=4, K=4, lda=4, ldc=4)
    a.update(HERK_BAD[info])
    A = np.zeros((4, 4), np.complex128); C = np.ones((4, 4), np.complex128, order="F")
    got = _capture(lambda: blx.cblas_zherk(102, a["uplo"], a["trans"], a["N"], a["K"], 1.0, A, a["lda"], 0.0, C,
                                           a["ldc"]))
    assert got == want
    assert np.all(C == 1.0) and blx.last_status() == blx.BLASX_ERR_ARG


@pytest.mark.parametrize("info,kw", [(2, dict(trans=112)), (9, dict(ldb=2)), (12, dict(ldc=2))])
def test_her2k_xerbla_matches_reference(blx, sgolden, info, kw):
    """ZHER2K reports under the reference's name for it, "ZHERK"."""
    want = [str(l) for l in sgolden["xerbla"] if str(l).startswith(f"cblas_zher2k|{info}|")][0].split("|", 2)[2]
    a = dict(trans=111, ldb=4, ldc=4)
    a.update(kw)
    A = np.zeros((4, 4), np.complex128); C = np.ones((4, 4), np.complex128, order="F")
    got = _capture(lambda: blx.cblas_zher2k(102, 121, a["trans"], 4, 4, 1.0, A, 4, A, a["ldb"], 0.0, C, a["ldc"]))
    assert got == want
    assert np.all(C == 1.0)


@pytest.mark.parametrize("up,tr", [("X", "N"), ("U", "Q"), ("U", "T")])
def test_f77_herk_errors_match_reference(blx, sgolden, up, tr):
    want = [str(l) for l in sgolden["xerbla"] if str(l).startswith(f"zherk_{up}{tr}|")][0].split("|", 2)[2]
    A = np.zeros((4, 4), np.complex128); C = np.ones((4, 4), np.complex128, order="F")
    got = _capture(lambda: blx.zherk_(up, tr, 4, 4, 1.0, A, 4, 0.0, C, 4))
    assert got == want
    assert np.all(C == 1.0)
