"""GPU tests of cblas_?herk / ?her2k (C/Z) and cblas_csyrk / csyr2k: the
reference's own outputs (golden fixtures, its CPU BLAS path; C holds NaN
outside its triangle and garbage imaginary parts on a Hermitian diagonal) on
the native and the emulated paths, larger problems against the double-double
oracle, in and out of core."""
import os

import numpy as np
import pytest

import oracle
from golden_cases import rank_k_case, rank_k_check
from test_symm_oracle import RANK_K, rank_k_keys

pytestmark = pytest.mark.gpu

GOLDEN_SYMM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "symm_trmm_golden.npz")


@pytest.fixture(scope="module")
def sgolden():
    return np.load(GOLDEN_SYMM)


@pytest.fixture(params=["native", "ozaki"])
def mode(blx, request):
    prev = blx.set_dgemm_mode(blx.MODE_NATIVE if request.param == "native" else blx.MODE_OZAKI)
    yield request.param
    blx.set_dgemm_mode(prev)


def run_rank_k(blx, kind, tag, x, al, be):
    C = x["C"].copy(order="F")
    fn = getattr(blx, f"cblas_{tag}{kind}")
    args = [x["order"], x["uplo"], x["trans"], x["N"], x["K"], al, x["A"], x["lda"]]
    if x["B"] is not None:
        args += [x["B"], x["ldb"]]
    fn(*args, be, C, x["ldc"])
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    return C


@pytest.mark.parametrize("prefix", RANK_K)
def test_matches_reference_outputs(blx, sgolden, mode, prefix):
    for key in rank_k_keys(sgolden, prefix):
        kind, tag, x, al, be, want = rank_k_case(sgolden, key)
        rank_k_check(x, run_rank_k(blx, kind, tag, x, al, be), want, al, be)


def herm_input(dt, N, uplo, seed):
    """C with NaN outside its uplo triangle and a nonzero imaginary diagonal."""
    C = oracle.uniform((N + 2, N), dt, seed)
    i, j = np.indices((N, N))
    C[:N, :N][(i > j) if uplo == "U" else (i < j)] = np.nan
    d = np.arange(N)
    C[d, d] = C[d, d].real + 0.5j
    return C


def check_herk(C, C0, uplo, trans, N, K, al, A, lda, be, B=None, ldb=None, seed=7):
    m = oracle.tri_mask(uplo, N)
    assert np.array_equal(C[:N, :N][~m], C0[:N, :N][~m], equal_nan=True)
    assert np.array_equal(C[N:], C0[N:])
    assert np.all(np.diag(C[:N, :N]).imag == 0)
    rng = np.random.default_rng(seed)
    ii = rng.integers(0, N, 6000); jj = rng.integers(0, N, 6000)
    keep = ((ii <= jj) if uplo == "U" else (ii >= jj)) & (ii != jj)
    ii, jj = ii[keep], jj[keep]
    ta, tb = ("N", "C") if trans == "N" else ("C", "N")
    C0r = np.nan_to_num(C0)
    if B is None:
        val, bound = oracle.dd_entries(ta, tb, N, N, K, al, A, lda, A, lda, be, C0r, N + 2, ii, jj)
    else:  # alpha A B^H + conj(alpha) B A^H + beta C0: the two halves of the sum
        v1, b1 = oracle.dd_entries(ta, tb, N, N, K, al, A, lda, B, ldb, be, C0r, N + 2, ii, jj)
        v2, b2 = oracle.dd_entries(ta, tb, N, N, K, np.conj(al), B, ldb, A, lda, 0.0, C0r, N + 2, ii, jj)
        val, bound = v1 + v2, b1 + b2
    ratio, err = oracle.componentwise_ratio(C, ii, jj, val, bound, K, C.dtype.type)
    assert ratio <= 1.0, ratio
    return err


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "C"])
@pytest.mark.parametrize("dt", [np.complex128, np.complex64])
def test_herk_large_vs_oracle(blx, mode, uplo, trans, dt):
    N, K = 900, 1100
    ra, ca = (N, K) if trans == "N" else (K, N)
    A = oracle.uniform((ra + 1, ca), dt, 21)
    C0 = herm_input(dt, N, uplo, 22)
    C = C0.copy(order="F")
    tag = "z" if dt == np.complex128 else "c"
    getattr(blx, f"cblas_{tag}herk")(102, blx.UPLO[uplo], blx.TRANS[trans], N, K, 1.25, A, ra + 1, -0.5, C, N + 2)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    assert blx.call_stats()["path"] == (2 if mode == "ozaki" else 1), blx.call_stats()
    check_herk(C, C0, uplo, trans, N, K, 1.25, A, ra + 1, -0.5)


@pytest.mark.parametrize("uplo,trans", [("U", "N"), ("L", "C")])
def test_zher2k_large_vs_oracle(blx, mode, uplo, trans):
    N, K = 700, 800
    ra, ca = (N, K) if trans == "N" else (K, N)
    A = oracle.uniform((ra, ca), np.complex128, 31)
    B = oracle.uniform((ra, ca), np.complex128, 32)
    C0 = herm_input(np.complex128, N, uplo, 33)
    C = C0.copy(order="F")
    al = complex(0.75, -0.5)
    blx.cblas_zher2k(102, blx.UPLO[uplo], blx.TRANS[trans], N, K, al, A, ra, B, ra, 0.25, C, N + 2)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    check_herk(C, C0, uplo, trans, N, K, al, A, ra, 0.25, B, ra)


@pytest.mark.parametrize("emulated", [False, True])
def test_zherk_out_of_core(blx, emulated):
    """A 64 MiB budget forces the tile cache: the diagonal tiles get their
    imaginary parts cleared before they are written back."""
    blx.set_hbm_budget(64 << 20)
    blx.set_tile(512)
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI if emulated else blx.MODE_NATIVE)
    try:
        N, K = 1700, 1300  # A (35 MB) and C (46 MB) exceed the budget together
        A = oracle.uniform((K, N), np.complex128, 41)
        C0 = herm_input(np.complex128, N, "L", 42)
        C = C0.copy(order="F")
        blx.cblas_zherk(102, 122, 113, N, K, 1.0, A, K, 0.5, C, N + 2)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        st = blx.call_stats()
        assert st["tile"] == 512 and st["path"] == (2 if emulated else 1), st
        check_herk(C, C0, "L", "C", N, K, 1.0, A, K, 0.5)
    finally:
        blx.set_hbm_budget(0)
        blx.set_tile(0)
        blx.set_dgemm_mode(prev)


def test_row_major_herk_is_the_transposed_problem(blx):
    N, K = 300, 200
    A = oracle.uniform((K, N), np.complex128, 51)  # row-major N x K = column-major K x N
    C0 = herm_input(np.complex128, N, "U", 52)[:N].copy(order="F")
    Crm, Ccm = C0.copy(order="F"), C0.copy(order="F")
    blx.cblas_zherk(101, 121, 111, N, K, 0.5, A, K, 2.0, Crm, N)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    blx.cblas_zherk(102, 122, 113, N, K, 0.5, A, K, 2.0, Ccm, N)
    np.testing.assert_array_equal(Crm, Ccm)


def test_f77_wrappers_match_cblas(blx):
    N, K = 260, 300
    A = oracle.uniform((N, K), np.complex64, 61)
    B = oracle.uniform((N, K), np.complex64, 62)
    C0 = herm_input(np.complex64, N, "U", 63)[:N].copy(order="F")
    C1, C2 = C0.copy(order="F"), C0.copy(order="F")
    blx.cblas_cher2k(102, 121, 111, N, K, complex(1, 2), A, N, B, N, 0.5, C1, N)
    blx.cher2k_("u", "N", N, K, complex(1, 2), A, N, B, N, 0.5, C2, N)
    assert np.array_equal(C1, C2, equal_nan=True)
    D1, D2 = C0.copy(order="F"), C0.copy(order="F")
    blx.cblas_csyrk(102, 121, 111, N, K, complex(0.5, -1), A, N, complex(2, 0), D1, N)
    blx.csyrk_("U", "N", N, K, complex(0.5, -1), A, N, complex(2, 0), D2, N)
    assert np.array_equal(D1, D2, equal_nan=True)
