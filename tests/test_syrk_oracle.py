"""CPU tests of the SYRK / SYR2K restatement in the oracle and of the
library's argument checking for them, both pinned to the reference: the
golden fixtures hold the reference's own outputs (its CPU BLAS path, which it
uses for every SYRK / SYR2K) and its xerbla_ lines (tests/golden/make_golden.py)."""
import numpy as np
import pytest

import oracle
from test_abi import _capture

UPLO = {121: "U", 122: "L"}
TR = {111: "N", 112: "T"}
DT = {"d": np.float64, "s": np.float32, "z": np.complex128}


def syrk_cases(golden, prefix):
    keys = sorted({k.rsplit("_", 1)[0] for k in golden.files if k.startswith(prefix)},
                  key=lambda k: int(k.split("_")[-1]))
    return keys


def regen_syrk(golden, key):
    tag = key.split("_")[1]
    dt = DT[tag]
    N, K, uplo, trans, lda, ldc, seed = (int(v) for v in golden[key + "_meta"])
    ra, ca = (N, K) if trans == 111 else (K, N)
    A = oracle.uniform((lda, ca), dt, seed)
    C0 = oracle.uniform((ldc, N), dt, seed + 1)
    assert np.allclose([np.sum(A), np.sum(C0)], golden[key + "_sum"]), "fixture generator changed"
    al, be = golden[key + "_scal"]
    if dt != np.complex128:
        al, be = al.real, be.real
    return dt, N, K, UPLO[uplo], TR[trans], A, lda, C0, ldc, al, be


def check_against_reference(C, Cref, C0, uplo, N, bound):
    m = oracle.tri_mask(uplo, N)
    # outside the triangle and beyond N rows: exactly the input
    untouched = ~m
    assert np.array_equal(C[:N, :N][untouched], C0[:N, :N][untouched])
    assert np.array_equal(C[N:, :], C0[N:, :])
    err = np.abs(C[:N, :N] - Cref[:N, :N])[m]
    assert np.all(err <= bound[m]), float(np.max(err / np.maximum(bound[m], 1e-300)))


def test_oracle_syrk_matches_reference(golden):
    keys = syrk_cases(golden, "syrk_")
    assert len(keys) == 48
    for key in keys:
        dt, N, K, uplo, trans, A, lda, C0, ldc, al, be = regen_syrk(golden, key)
        C = oracle.syrk(uplo, trans, N, K, al, A, lda, be, C0.copy(order="F"), ldc)
        opA = A[:N, :K] if trans == "N" else A[:K, :N].T
        u = {np.float64: 2.0 ** -53, np.float32: 2.0 ** -24, np.complex128: 2.0 ** -53}[dt]
        g = 2 * (K + 2) * u * (2.0 if dt == np.complex128 else 1.0)  # both sides' roundings
        bound = g * (abs(al) * (np.abs(opA).astype(np.float64) @ np.abs(opA.T).astype(np.float64))
                     + abs(be) * np.abs(C0[:N, :N]).astype(np.float64))
        check_against_reference(C, golden[key + "_C"], C0, uplo, N, bound)


def test_oracle_syr2k_matches_reference(golden):
    keys = syrk_cases(golden, "syr2k_")
    assert len(keys) == 8
    for key in keys:
        N, K, uplo, trans, ld, ldc, seed = (int(v) for v in golden[key + "_meta"])
        ra, ca = (N, K) if trans == 111 else (K, N)
        A = oracle.uniform((ra, ca), np.float64, seed)
        B = oracle.uniform((ra, ca), np.float64, seed + 1)
        C0 = oracle.uniform((N, N), np.float64, seed + 2)
        assert np.allclose([np.sum(A), np.sum(B), np.sum(C0)], golden[key + "_sum"])
        C = oracle.syrk(UPLO[uplo], TR[trans], N, K, 1.5, A, ra, -0.25, C0.copy(order="F"), N, B=B, ldb=ra)
        opA = A if trans == 111 else A.T
        opB = B if trans == 111 else B.T
        bound = 2 * (K + 3) * 2.0 ** -53 * (1.5 * (np.abs(opA) @ np.abs(opB.T) + np.abs(opB) @ np.abs(opA.T))
                                           + 0.25 * np.abs(C0))
        check_against_reference(C, golden[key + "_C"], C0, UPLO[uplo], N, bound)


BAD = {1: dict(uplo=999), 2: dict(trans=999), 3: dict(N=-1), 4: dict(K=-1), 7: dict(lda=2), 10: dict(ldc=2)}


@pytest.mark.parametrize("info", sorted(BAD))
def test_syrk_xerbla_matches_reference(blx, golden, info):
    want = [str(l) for l in golden["xerbla"] if str(l).startswith(f"cblas_dsyrk|{info}|")][0].split("|", 2)[2]
    a = dict(uplo=121, trans=111, N=4, K=4, lda=4, ldc=4)
    a.update(BAD[info])
    A = np.zeros((4, 4)); C = np.ones((4, 4), order="F")
    got = _capture(lambda: blx.cblas_dsyrk(102, a["uplo"], a["trans"], a["N"], a["K"], 1.0, A, a["lda"], 0.0, C,
                                           a["ldc"]))
    assert got == want
    assert np.all(C == 1.0) and blx.last_status() == blx.BLASX_ERR_ARG


@pytest.mark.parametrize("info,kw", [(7, dict(lda=2)), (9, dict(ldb=2)), (12, dict(ldc=2))])
def test_syr2k_xerbla_matches_reference(blx, golden, info, kw):
    want = [str(l) for l in golden["xerbla"] if str(l).startswith(f"cblas_dsyr2k|{info}|")][0].split("|", 2)[2]
    a = dict(lda=4, ldb=4, ldc=4)
    a.update(kw)
    A = np.zeros((4, 4)); C = np.ones((4, 4), order="F")
    got = _capture(lambda: blx.cblas_dsyr2k(102, 121, 111, 4, 4, 1.0, A, a["lda"], A, a["ldb"], 0.0, C, a["ldc"]))
    assert got == want
    assert np.all(C == 1.0)


@pytest.mark.parametrize("up,tr", [("X", "N"), ("U", "Q"), ("X", "Q")])
def test_f77_syrk_errors_match_reference(blx, golden, up, tr):
    want = [str(l) for l in golden["xerbla"] if str(l).startswith(f"dsyrk_{up}{tr}|")][0].split("|", 2)[2]
    A = np.zeros((4, 4)); C = np.ones((4, 4), order="F")
    got = _capture(lambda: blx.dsyrk_(up, tr, 4, 4, 1.0, A, 4, 0.0, C, 4))
    assert got == want
    assert np.all(C == 1.0)


def test_zsyrk_conjtrans_is_illegal(blx):
    A = np.zeros((4, 4), np.complex128); C = np.ones((4, 4), np.complex128, order="F")
    out = _capture(lambda: blx.cblas_zsyrk(102, 121, 113, 4, 4, 1.0, A, 4, 0.0, C, 4))
    assert "ZSYRK  parameter number  2" in out and np.all(C == 1.0)


def test_syrk_quick_return_needs_no_gpu(blx):
    C = np.ones((4, 4), order="F")
    blx.cblas_dsyrk(102, 121, 111, 0, 4, 1.0, C, 4, 0.0, C, 4)
    assert blx.last_status() == blx.BLASX_OK and np.all(C == 1.0)
