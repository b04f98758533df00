"""GPU tests of cblas_?symm / ?hemm / ?trmm / ?trsm: the reference's own outputs
(golden fixtures, its CPU BLAS path; the entries BLAS must not read hold NaN)
on the native and the emulated paths, larger cases against the double-double
oracle, and the F77 wrappers."""
import os

import numpy as np
import pytest

import oracle
from golden_cases import symm_case, symm_check, symm_keys

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


def run_case(blx, kind, tag, x, al, be):
    """The library call the reference made for this case; returns the output array."""
    if kind in "SH":
        C = x["C"].copy(order="F")
        fn = getattr(blx, f"cblas_{tag}{'symm' if kind == 'S' else 'hemm'}")
        fn(x["order"], x["side"], x["uplo"], x["M"], x["N"], al, x["A"], x["lda"], x["B"], x["ldb"], be, C,
           x["ldc"])
        out = C
    else:
        out = x["B"].copy(order="F")
        getattr(blx, f"cblas_{tag}{'trmm' if kind == 'T' else 'trsm'}")(
            x["order"], x["side"], x["uplo"], x["trans"], x["diag"], x["M"], x["N"], al, x["A"], x["lda"], out,
            x["ldb"])
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    return out


@pytest.mark.parametrize("prefix", ["symm_", "hemm_", "trmm_", "trsm_"])
def test_matches_reference_outputs(blx, sgolden, mode, prefix):
    for key in symm_keys(sgolden, prefix):
        kind, tag, x, al, be, want = symm_case(sgolden, key)
        got = run_case(blx, kind, tag, x, al, be)
        symm_check(kind, x, got, want, al, be)


def sample(M, N, seed, n=5000):
    rng = np.random.default_rng(seed)
    return rng.integers(0, M, n), rng.integers(0, N, n)


def check_dd(C, ta, tb, M, N, K, al, X, ldx, Y, ldy, be, C0, ldc, seed):
    ii, jj = sample(M, N, seed)
    val, bound = oracle.dd_entries(ta, tb, M, N, K, al, X, ldx, Y, ldy, be, C0, ldc, ii, jj)
    ratio, err = oracle.componentwise_ratio(C, ii, jj, val, bound, K, C.dtype.type)
    assert ratio <= 1.0, ratio
    return err


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("dt,herm", [(np.float64, False), (np.complex128, False), (np.complex128, True)])
def test_symm_large_vs_oracle(blx, mode, side, uplo, dt, herm):
    """Larger than one tile, ragged; A's other triangle is NaN. The emulated
    path is at least as accurate as the native kernel on the same inputs."""
    M, N = 1100, 900
    na = M if side == "L" else N
    A = oracle.uniform((na + 3, na), dt, 11)
    i, j = np.indices((na, na))
    A[:na, :na][(i > j) if uplo == "U" else (i < j)] = np.nan
    B = oracle.uniform((M + 1, N), dt, 12)
    C0 = oracle.uniform((M + 2, N), dt, 13)
    al, be = (1.25, -0.5) if dt == np.float64 else (complex(1.25, 0.5), complex(-0.5, 0.25))
    tag = "d" if dt == np.float64 else "z"
    fn = getattr(blx, f"cblas_{tag}{'hemm' if herm else 'symm'}")

    def call():
        C = C0.copy(order="F")
        fn(102, blx.SIDE[side], blx.UPLO[uplo], M, N, al, A, na + 3, B, M + 1, be, C, M + 2)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        return C

    C = call()
    assert blx.call_stats()["path"] == (2 if mode == "ozaki" else 1), blx.call_stats()
    assert np.array_equal(C[M:], C0[M:])
    Af = oracle.complete("H" if herm else "S", uplo, A, na)
    args = (Af, na, B, M + 1) if side == "L" else (B, M + 1, Af, na)
    err = check_dd(C, "N", "N", M, N, na, al, *args, be, C0, M + 2, 21)
    if mode == "ozaki":
        blx.set_dgemm_mode(blx.MODE_NATIVE)
        Cn = call()
        blx.set_dgemm_mode(blx.MODE_OZAKI)
        err_n = check_dd(Cn, "N", "N", M, N, na, al, *args, be, C0, M + 2, 21)
        assert err <= max(err_n, 2.0 ** -53), (err, err_n)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo,trans,diag", [("U", "N", "N"), ("L", "T", "U"), ("U", "C", "U"), ("L", "N", "N")])
@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_trmm_large_vs_oracle(blx, mode, side, uplo, trans, diag, dt):
    """B = alpha op(A) B in place, A's other triangle (and a unit diagonal) NaN."""
    if trans == "C" and dt == np.float64:
        trans = "T"
    M, N = 1000, 1300
    na = M if side == "L" else N
    A = oracle.uniform((na, na), dt, 31)
    i, j = np.indices((na, na))
    A[(i > j) if uplo == "U" else (i < j)] = np.nan
    if diag == "U":
        np.fill_diagonal(A, np.nan)
    B0 = oracle.uniform((M + 1, N), dt, 32)
    B = B0.copy(order="F")
    al = 0.75 if dt == np.float64 else complex(0.75, -0.5)
    tag = "d" if dt == np.float64 else "z"
    getattr(blx, f"cblas_{tag}trmm")(102, blx.SIDE[side], blx.UPLO[uplo], blx.TRANS[trans], blx.DIAG[diag], M, N,
                                     al, A, na, B, M + 1)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    assert blx.call_stats()["path"] == (2 if mode == "ozaki" else 1), blx.call_stats()
    assert np.array_equal(B[M:], B0[M:])
    Af = oracle.complete("T", uplo, A, na, diag)
    Z = np.zeros_like(B0)
    if side == "L":
        check_dd(B, trans, "N", M, N, M, al, Af, na, B0, M + 1, 0.0, Z, M + 1, 41)
    else:
        check_dd(B, "N", trans, M, N, N, al, B0, M + 1, Af, na, 0.0, Z, M + 1, 41)


def test_f77_wrappers_match_cblas(blx):
    M, N = 300, 200
    A = oracle.uniform((M, M), np.float64, 51)
    B = oracle.uniform((M, N), np.float64, 52)
    C0 = oracle.uniform((M, N), np.float64, 53)
    C1, C2 = C0.copy(order="F"), C0.copy(order="F")
    blx.cblas_dsymm(102, 141, 122, M, N, 0.5, A, M, B, M, 2.0, C1, M)
    blx.dsymm_("l", "L", M, N, 0.5, A, M, B, M, 2.0, C2, M)
    assert np.array_equal(C1, C2)
    Az = oracle.uniform((N, N), np.complex128, 54)
    Bz = oracle.uniform((M, N), np.complex128, 55)
    B1, B2 = Bz.copy(order="F"), Bz.copy(order="F")
    blx.cblas_ztrmm(102, 142, 121, 113, 132, M, N, complex(1, 2), Az, N, B1, M)
    blx.ztrmm_("R", "u", "c", "U", M, N, complex(1, 2), Az, N, B2, M)
    assert np.array_equal(B1, B2)
    Ac = oracle.uniform((M, M), np.complex64, 56)
    Bc = oracle.uniform((M, N), np.complex64, 57)
    Cc0 = oracle.uniform((M, N), np.complex64, 58)
    D1, D2 = Cc0.copy(order="F"), Cc0.copy(order="F")
    blx.cblas_chemm(102, 141, 121, M, N, complex(0.5, 0.5), Ac, M, Bc, M, complex(1, 0), D1, M)
    blx.chemm_("L", "U", M, N, complex(0.5, 0.5), Ac, M, Bc, M, complex(1, 0), D2, M)
    assert np.array_equal(D1, D2)


def test_symm_while_serving(blx):
    blx.serve_start(0, 0, 4)
    try:
        M, N = 700, 500
        A = oracle.uniform((M, M), np.float64, 71)
        B = oracle.uniform((M, N), np.float64, 72)
        C0 = oracle.uniform((M, N), np.float64, 73)
        C = C0.copy(order="F")
        blx.cblas_dsymm(102, 141, 121, M, N, 1.0, A, M, B, M, 1.0, C, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    finally:
        blx.serve_stop()
    want = oracle.symm("L", "U", M, N, 1.0, A, M, B, M, 1.0, C0.copy(order="F"), M)
    np.testing.assert_allclose(C, want, rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("dt", [np.float32, np.complex64, np.float64])
@pytest.mark.parametrize("side,uplo", [("R", "L"), ("L", "U")])
def test_trmm_emulated_is_componentwise_accurate_at_the_tip(blx, dt, side, uplo):
    """Emulated path with the triangle wider than one diagonal block: the
    diagonal blocks run natively, so the tip of a unit triangle (one nonzero,
    the 1) reproduces alpha B exactly, and for the single-precision types every
    entry is within the componentwise bound of the exact product."""
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI)
    try:
        M, N = 600, 700
        na = M if side == "L" else N
        A = oracle.uniform((na, na), dt, 91)
        B0 = oracle.uniform((M, N), dt, 92)
        B = B0.copy(order="F")
        tag = {np.float32: "s", np.complex64: "c", np.float64: "d"}[dt]
        getattr(blx, f"cblas_{tag}trmm")(102, blx.SIDE[side], blx.UPLO[uplo], 111, 132, M, N, 0.5, A, na, B, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert blx.call_stats()["path"] == 2, blx.call_stats()
        if side == "R":  # lower, unit: the last column of A is e_N
            assert np.array_equal(B[:, -1], (0.5 * B0[:, -1]).astype(dt))
        else:  # upper, unit: the last row of A is e_M^T
            assert np.array_equal(B[-1, :], (0.5 * B0[-1, :]).astype(dt))
        Af = oracle.complete("T", uplo, A, na, "U")
        if dt == np.float64:
            Z = np.zeros_like(B0)
            if side == "L":
                check_dd(B, "N", "N", M, N, M, 0.5, Af, na, B0, M, 0.0, Z, M, 93)
            else:
                check_dd(B, "N", "N", M, N, N, 0.5, B0, M, Af, na, 0.0, Z, M, 93)
            return
        wide = np.complex128 if dt == np.complex64 else np.float64
        exact = 0.5 * (Af.astype(wide) @ B0.astype(wide) if side == "L" else B0.astype(wide) @ Af.astype(wide))
        aA, aB = np.abs(Af).astype(np.float64), np.abs(B0).astype(np.float64)
        scale = 0.5 * (aA @ aB if side == "L" else aB @ aA)
        bound = (na + 2) * 2.0 ** -24 * (2.0 if dt == np.complex64 else 1.0) * scale
        err = np.abs(B.astype(wide) - exact)
        assert np.all(err <= bound), float(np.max(err / np.maximum(bound, 1e-300)))
    finally:
        blx.set_dgemm_mode(prev)


def dominant_triangle(dt, na, uplo, diag, seed):
    """A well-conditioned triangle (off-diagonal U[-1, 1] / na, diagonal 2 +
    U[-1, 1] / na) with NaN in every entry BLAS must not read."""
    A = oracle.uniform((na, na), dt, seed) / na
    A[np.arange(na), np.arange(na)] += 2
    i, j = np.indices((na, na))
    A[(i > j) if uplo == "U" else (i < j)] = np.nan
    if diag == "U":
        np.fill_diagonal(A, np.nan)
    return A


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo,trans,diag", [("U", "N", "N"), ("L", "T", "U"), ("U", "C", "N"), ("L", "N", "U")])
@pytest.mark.parametrize("dt", [np.float64, np.complex128, np.float32, np.complex64])
def test_trsm_large_backward_error(blx, mode, side, uplo, trans, diag, dt):
    """B := alpha op(A)^-1 B (or B op(A)^-1), 1000 x 1300 with ragged leading
    dimensions (recursion down to ragged 64-row leaves): the residual
    op(A) X - alpha B of sampled entries, in double-double, is within
    2 (K + 2) u (|op(A)| |X| + |alpha| |B|)."""
    if trans == "C" and dt in (np.float64, np.float32):
        trans = "T"
    M, N = 1000, 1300
    na = M if side == "L" else N
    A = dominant_triangle(dt, na, uplo, diag, 31)
    B0 = oracle.uniform((M + 1, N), dt, 32)
    B = B0.copy(order="F")
    al = 0.75 if dt in (np.float64, np.float32) else complex(0.75, -0.5)
    tag = {np.float64: "d", np.complex128: "z", np.float32: "s", np.complex64: "c"}[dt]
    getattr(blx, f"cblas_{tag}trsm")(102, blx.SIDE[side], blx.UPLO[uplo], blx.TRANS[trans], blx.DIAG[diag], M, N,
                                     al, A, na, B, M + 1)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    st = blx.call_stats()
    if mode == "ozaki":
        assert st["path"] == 2, st
    assert np.array_equal(B[M:], B0[M:]) and np.all(np.isfinite(B))
    Af = oracle.complete("T", uplo, A, na, diag)
    ii, jj = sample(M, N, 43)
    if side == "L":
        val, bound = oracle.dd_entries(trans, "N", M, N, M, 1.0, Af, na, B, M + 1, -al, B0, M + 1, ii, jj)
    else:
        val, bound = oracle.dd_entries("N", trans, M, N, N, 1.0, B, M + 1, Af, na, -al, B0, M + 1, ii, jj)
    u = oracle.UNIT_ROUNDOFF[np.dtype(dt).type] * (2.0 if np.issubdtype(dt, np.complexfloating) else 1.0)
    ratio = np.max(np.abs(val) / (2 * (na + 2) * u * bound))
    assert ratio <= 1.0, ratio


def test_trsm_row_major_is_the_transposed_problem(blx):
    M, N = 300, 200
    A = dominant_triangle(np.float64, M, "U", "N", 61)
    B = oracle.uniform((N, M), np.float64, 62)  # row-major M x N = column-major N x M
    Brm, Bcm = B.copy(order="F"), B.copy(order="F")
    blx.cblas_dtrsm(101, 141, 121, 111, 131, M, N, 1.5, A.T.copy(order="F"), M, Brm, N)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    blx.cblas_dtrsm(102, 142, 122, 111, 131, N, M, 1.5, A.T.copy(order="F"), M, Bcm, N)
    np.testing.assert_array_equal(Brm, Bcm)


def test_trsm_alpha_zero_sets_b_to_zero_without_reading_a(blx):
    M, N = 100, 70
    A = np.full((M, M), np.nan, order="F")
    B = oracle.uniform((M, N), np.float64, 63)
    blx.cblas_dtrsm(102, 141, 121, 111, 131, M, N, 0.0, A, M, B, M)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    assert np.all(B == 0.0) and blx.call_stats()["path"] == 3


def test_trsm_f77_matches_cblas(blx):
    M, N = 500, 300
    A = dominant_triangle(np.complex128, N, "L", "N", 64)
    B0 = oracle.uniform((M, N), np.complex128, 65)
    B1, B2 = B0.copy(order="F"), B0.copy(order="F")
    blx.cblas_ztrsm(102, 142, 122, 113, 131, M, N, complex(1, -1), A, N, B1, M)
    blx.ztrsm_("r", "L", "C", "n", M, N, complex(1, -1), A, N, B2, M)
    assert np.array_equal(B1, B2)


@pytest.mark.parametrize("side,uplo,dt,herm", [("L", "U", np.float64, False), ("R", "L", np.float64, False),
                                                ("L", "L", np.complex128, True), ("R", "U", np.complex128, True)])
@pytest.mark.parametrize("emulated", [False, True])
def test_symm_out_of_core(blx, side, uplo, dt, herm, emulated):
    """A 64 MiB budget forces the tile cache: tiles of the unstored triangle
    (NaN here) are read from the stored one across the diagonal, diagonal
    tiles are completed on arrival."""
    blx.set_hbm_budget(64 << 20)
    blx.set_tile(512)
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI if emulated else blx.MODE_NATIVE)
    try:
        M, N = (2000, 1800) if dt == np.float64 else (1500, 1400)  # A, B, C exceed the budget together
        na = M if side == "L" else N
        A = oracle.uniform((na + 1, na), dt, 81)
        i, j = np.indices((na, na))
        A[:na, :na][(i > j) if uplo == "U" else (i < j)] = np.nan
        if herm:
            d = np.arange(na)
            A[d, d] = A[d, d].real + 0.25j  # imaginary parts of a Hermitian diagonal are not read
        B = oracle.uniform((M, N), dt, 82)
        C0 = oracle.uniform((M, N), dt, 83)
        C = C0.copy(order="F")
        al, be = (0.75, 0.5) if dt == np.float64 else (complex(0.75, 0.25), complex(0.5, -0.5))
        fn = getattr(blx, f"cblas_{'z' if herm else 'd'}{'hemm' if herm else 'symm'}")
        fn(102, blx.SIDE[side], blx.UPLO[uplo], M, N, al, A, na + 1, B, M, be, C, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        st = blx.call_stats()
        assert st["tile"] == 512 and st["path"] == (2 if emulated else 1), st
        Af = oracle.complete("H" if herm else "S", uplo, A, na)
        args = (Af, na, B, M) if side == "L" else (B, M, Af, na)
        check_dd(C, "N", "N", M, N, na, al, *args, be, C0, M, 85)
    finally:
        blx.set_hbm_budget(0)
        blx.set_tile(0)
        blx.set_dgemm_mode(prev)


@pytest.mark.parametrize("fn", ["trsm", "trmm"])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "N"), ("U", "N", "U"), ("L", "T", "N")])
def test_tri_streams_the_order_in_blocks(blx, mode, fn, side, uplo, trans, diag):
    """An order of 6200 is copied, solved or multiplied and copied back in
    blocks: three of 2304 for the solve, five of 1280 for the multiply (the
    last ragged), ascending or descending with the substitution order (both
    occur on each side); the result is within the backward-error bound
    (solve) or the componentwise bound (multiply)."""
    K, nv = 6200, 96
    M, N = (K, nv) if side == "L" else (nv, K)
    A = dominant_triangle(np.float64, K, uplo, diag, 111)
    B0 = oracle.uniform((M + 1, N), np.float64, 112)
    B = B0.copy(order="F")
    getattr(blx, f"cblas_d{fn}")(102, blx.SIDE[side], blx.UPLO[uplo], blx.TRANS[trans], blx.DIAG[diag], M, N, 0.75,
                                 A, K, B, M + 1)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    st = blx.call_stats()
    assert st["tile"] == (1280 if fn == "trmm" else 2304) and st["path"] == (2 if mode == "ozaki" else 1), st
    assert np.array_equal(B[M:], B0[M:]) and np.all(np.isfinite(B))
    Af = oracle.complete("T", uplo, A, K, diag)
    if fn == "trmm":
        Z = np.zeros_like(B0)
        if side == "L":
            check_dd(B, trans, "N", M, N, K, 0.75, Af, K, B0, M + 1, 0.0, Z, M + 1, 113)
        else:
            check_dd(B, "N", trans, M, N, K, 0.75, B0, M + 1, Af, K, 0.0, Z, M + 1, 113)
        return
    ii, jj = sample(M, N, 114)
    if side == "L":
        val, bound = oracle.dd_entries(trans, "N", M, N, K, 1.0, Af, K, B, M + 1, -0.75, B0, M + 1, ii, jj)
    else:
        val, bound = oracle.dd_entries("N", trans, M, N, K, 1.0, B, M + 1, Af, K, -0.75, B0, M + 1, ii, jj)
    assert np.max(np.abs(val) / (2 * (K + 2) * 2.0 ** -53 * bound)) <= 1.0


@pytest.mark.parametrize("emulated", [False, True])
def test_trsm_streams_b_beyond_the_budget(blx, emulated):
    """B (74 MB) does not fit a 48 MiB budget beside A (8 MB): its columns
    stream through two device panels while A stays resident; the residual
    of every panel is within the backward-error bound."""
    blx.set_hbm_budget(48 << 20)
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI if emulated else blx.MODE_NATIVE)
    try:
        M, N = 1024, 9000
        A = dominant_triangle(np.float64, M, "L", "N", 71)
        B0 = oracle.uniform((M, N), np.float64, 72)
        B = B0.copy(order="F")
        blx.cblas_dtrsm(102, 141, 122, 111, 131, M, N, 0.5, A, M, B, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        st = blx.call_stats()
        assert 0 < st["tile"] < N and st["path"] == (2 if emulated else 1), st
        Af = oracle.complete("T", "L", A, M, "N")
        ii, jj = sample(M, N, 73)
        jj[:3] = [0, N - 1, st["tile"]]  # both ends and a panel boundary
        val, bound = oracle.dd_entries("N", "N", M, N, M, 1.0, Af, M, B, M, -0.5, B0, M, ii, jj)
        assert np.max(np.abs(val) / (2 * (M + 2) * 2.0 ** -53 * bound)) <= 1.0
    finally:
        blx.set_hbm_budget(0)
        blx.set_dgemm_mode(prev)


def test_trmm_streams_b_rows_beyond_the_budget(blx):
    """A right multiply streams B by rows: ZTRMM with B 48 MB under a 32 MiB budget."""
    blx.set_hbm_budget(32 << 20)
    try:
        M, N = 5000, 600
        A = oracle.uniform((N, N), np.complex128, 81)
        i, j = np.indices((N, N))
        A[i < j] = np.nan  # lower: the upper triangle is not read
        B0 = oracle.uniform((M, N), np.complex128, 82)
        B = B0.copy(order="F")
        al = complex(0.5, -0.25)
        blx.cblas_ztrmm(102, 142, 122, 113, 131, M, N, al, A, N, B, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert 0 < blx.call_stats()["tile"] < M
        Af = oracle.complete("T", "L", A, N, "N")
        check_dd(B, "N", "C", M, N, N, al, B0, M, Af, N, 0.0, np.zeros_like(B0), M, 83)
    finally:
        blx.set_hbm_budget(0)


@pytest.mark.parametrize("fn", ["trsm", "trmm"])
@pytest.mark.parametrize("side,uplo,trans,diag", [("L", "L", "N", "N"), ("L", "U", "T", "U"), ("R", "U", "N", "N"),
                                                  ("R", "L", "T", "N")])
def test_tri_halves_an_a_beyond_the_budget(blx, mode, fn, side, uplo, trans, diag):
    """A of order 1700 (23 MB) under a 12 MiB budget with 256-edge tiles: the
    order is halved on the host (pieces of at most 1024, some halved again),
    the off-diagonal blocks run as host GEMMs through the tile cache, and the
    result is within the backward-error bound (solve) or the componentwise
    bound (multiply); B's padding rows are not touched."""
    blx.set_hbm_budget(12 << 20)
    blx.set_tile(256)
    try:
        K, nv = 1700, 300
        M, N = (K, nv) if side == "L" else (nv, K)
        A = dominant_triangle(np.float64, K, uplo, diag, 121)
        B0 = oracle.uniform((M + 1, N), np.float64, 122)
        B = B0.copy(order="F")
        getattr(blx, f"cblas_d{fn}")(102, blx.SIDE[side], blx.UPLO[uplo], blx.TRANS[trans], blx.DIAG[diag], M, N,
                                     0.75, A, K, B, M + 1)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        st = blx.call_stats()
        assert 0 < st["tile"] <= 1024 and st["path"] == (2 if mode == "ozaki" else 1), st
        assert st["h2d_bytes"] > 0 and st["d2h_bytes"] > 0
    finally:
        blx.set_hbm_budget(0)
        blx.set_tile(0)
    assert np.array_equal(B[M:], B0[M:]) and np.all(np.isfinite(B))
    Af = oracle.complete("T", uplo, A, K, diag)
    if fn == "trmm":
        Z = np.zeros_like(B0)
        if side == "L":
            check_dd(B, trans, "N", M, N, K, 0.75, Af, K, B0, M + 1, 0.0, Z, M + 1, 123)
        else:
            check_dd(B, "N", trans, M, N, K, 0.75, B0, M + 1, Af, K, 0.0, Z, M + 1, 123)
        return
    ii, jj = sample(M, N, 124)
    if side == "L":
        val, bound = oracle.dd_entries(trans, "N", M, N, K, 1.0, Af, K, B, M + 1, -0.75, B0, M + 1, ii, jj)
    else:
        val, bound = oracle.dd_entries("N", trans, M, N, K, 1.0, B, M + 1, Af, K, -0.75, B0, M + 1, ii, jj)
    assert np.max(np.abs(val) / (2 * (K + 2) * 2.0 ** -53 * bound)) <= 1.0


def test_tri_beyond_the_budget(blx):
    """alpha = 0 streams zeros into B without reading A. An A beyond a 4 MB
    budget is halved on the host only when the halves' update GEMM can run:
    with the default tile edge (4096) it cannot, the call is refused before
    any work and B is left unchanged."""
    blx.set_hbm_budget(4 << 20)
    try:
        M, N = 1024, 1024  # A alone is 8 MB
        A = np.full((M, M), np.nan, order="F")
        B = oracle.uniform((M, N), np.float64, 91)
        blx.cblas_dtrsm(102, 141, 121, 111, 131, M, N, 0.0, A, M, B, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        assert np.all(B == 0.0)
        A = oracle.uniform((M, M), np.float64, 92)
        B0 = oracle.uniform((M, N), np.float64, 93)
        B = B0.copy(order="F")
        blx.cblas_dtrmm(102, 141, 121, 111, 131, M, N, 1.0, A, M, B, M)
        assert blx.last_status() == blx.BLASX_ERR_UNSUPPORTED
        assert np.array_equal(B, B0)
    finally:
        blx.set_hbm_budget(0)


@pytest.mark.parametrize("fn", ["trmm", "trsm"])
@pytest.mark.parametrize("mode", ["native", "ozaki"])
def test_device_entries_match_host(blx, fn, mode):
    """blasx_dtrmm_device / blasx_dtrsm_device on device pointers give the
    host call's result (the other triangle of A holds NaN)."""
    torch = pytest.importorskip("torch")
    prev = blx.set_dgemm_mode(blx.MODE_NATIVE if mode == "native" else blx.MODE_OZAKI)
    try:
        M, N = 700, 900
        A = dominant_triangle(np.float64, M, "U", "N", 101)
        B0 = oracle.uniform((M, N), np.float64, 102)
        Bh = B0.copy(order="F")
        getattr(blx, f"cblas_d{fn}")(102, 141, 121, 111, 131, M, N, 0.5, A, M, Bh, M)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        dA = torch.from_numpy(A.T.copy()).cuda()
        dB = torch.from_numpy(B0.T.copy()).cuda()
        s = torch.cuda.Stream(); s.wait_stream(torch.cuda.current_stream())
        rc = getattr(blx, f"d{fn}_device")("L", "U", "N", "N", M, N, 0.5, dA, M, dB, M, stream=s)
        assert rc == 0, blx.last_error()
        torch.cuda.synchronize()
        np.testing.assert_allclose(dB.cpu().numpy().T, Bh, rtol=1e-12, atol=1e-12)
    finally:
        blx.set_dgemm_mode(prev)
