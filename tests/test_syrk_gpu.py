"""GPU tests of cblas_?syrk / ?syr2k: the reference's own outputs (golden
fixtures, its CPU BLAS path) and the double-double oracle, on the native and
the emulated paths; the triangle outside uplo (and rows beyond N) must come
back bit for bit unchanged."""
import numpy as np
import pytest

import oracle
from test_syrk_oracle import DT, TR, UPLO, check_against_reference, regen_syrk, syrk_cases

pytestmark = pytest.mark.gpu

MODES = ["native", "ozaki"]


@pytest.fixture(params=MODES)
def mode(blx, request):
    prev = blx.set_dgemm_mode(blx.MODE_NATIVE if request.param == "native" else blx.MODE_OZAKI)
    yield request.param
    blx.set_dgemm_mode(prev)


def call_syrk(blx, dt, uplo, trans, N, K, al, A, lda, be, C, ldc, order=102):
    fn = {np.float64: blx.cblas_dsyrk, np.float32: blx.cblas_ssyrk, np.complex128: blx.cblas_zsyrk}[dt]
    fn(order, {"U": 121, "L": 122}[uplo], {"N": 111, "T": 112}[trans], N, K, al, A, lda, be, C, ldc)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    return blx.call_stats()


def tri_bound(dt, K, al, be, opA, opB, C0):
    u = {np.float64: 2.0 ** -53, np.float32: 2.0 ** -24, np.complex128: 2.0 ** -53}[dt]
    g = 2 * (K + 2) * u * (2.0 if dt == np.complex128 else 1.0)
    return g * (abs(al) * (np.abs(opA).astype(np.float64) @ np.abs(opB).astype(np.float64))
                + abs(be) * np.abs(C0).astype(np.float64))


def test_syrk_matches_reference_outputs(blx, golden, mode):
    for key in syrk_cases(golden, "syrk_"):
        dt, N, K, uplo, trans, A, lda, C0, ldc, al, be = regen_syrk(golden, key)
        C = C0.copy(order="F")
        call_syrk(blx, dt, uplo, trans, N, K, al, A, lda, be, C, ldc)
        opA = A[:N, :K] if trans == "N" else A[:K, :N].T
        check_against_reference(C, golden[key + "_C"], C0, uplo, N, tri_bound(dt, K, al, be, opA, opA.T, C0[:N, :N]))


def test_syr2k_matches_reference_outputs(blx, golden, mode):
    for key in syrk_cases(golden, "syr2k_"):
        N, K, up, tr, ld, ldc, seed = (int(v) for v in golden[key + "_meta"])
        ra, ca = (N, K) if tr == 111 else (K, N)
        A = oracle.uniform((ra, ca), np.float64, seed)
        B = oracle.uniform((ra, ca), np.float64, seed + 1)
        C0 = oracle.uniform((N, N), np.float64, seed + 2)
        C = C0.copy(order="F")
        blx.cblas_dsyr2k(102, up, tr, N, K, 1.5, A, ra, B, ra, -0.25, C, N)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        opA, opB = (A, B) if tr == 111 else (A.T, B.T)
        bound = 2 * (K + 3) * 2.0 ** -53 * (1.5 * (np.abs(opA) @ np.abs(opB.T) + np.abs(opB) @ np.abs(opA.T))
                                           + 0.25 * np.abs(C0))
        check_against_reference(C, golden[key + "_C"], C0, UPLO[up], N, bound)


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_dsyrk_large_vs_oracle(blx, mode, uplo, trans):
    """Larger than one tile in both dimensions, ragged; the emulated path slices
    A once for both operands. The emulation must be at least as accurate as
    the native kernel on the same inputs."""
    N, K = 1100, 1500
    ra, ca = (N, K) if trans == "N" else (K, N)
    A = oracle.uniform((ra + 3, ca), np.float64, 41)
    C0 = oracle.uniform((N + 2, N), np.float64, 42)
    C = C0.copy(order="F")
    st = call_syrk(blx, np.float64, uplo, trans, N, K, 1.25, A, ra + 3, -0.5, C, N + 2)
    assert st["path"] == (2 if mode == "ozaki" else 1), st
    m = oracle.tri_mask(uplo, N)
    assert np.array_equal(C[:N, :N][~m], C0[:N, :N][~m]) and np.array_equal(C[N:], C0[N:])
    rng = np.random.default_rng(5)
    ii = rng.integers(0, N, 6000); jj = rng.integers(0, N, 6000)
    keep = (ii <= jj) if uplo == "U" else (ii >= jj)
    ii, jj = ii[keep], jj[keep]
    ta, tb = ("N", "T") if trans == "N" else ("T", "N")
    val, bound = oracle.dd_entries(ta, tb, N, N, K, 1.25, A, ra + 3, A, ra + 3, -0.5, C0, N + 2, ii, jj)
    ratio, err = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float64)
    assert ratio <= 1.0
    if mode == "ozaki":
        blx.set_dgemm_mode(blx.MODE_NATIVE)
        Cn = C0.copy(order="F")
        call_syrk(blx, np.float64, uplo, trans, N, K, 1.25, A, ra + 3, -0.5, Cn, N + 2)
        blx.set_dgemm_mode(blx.MODE_OZAKI)
        _, err_n = oracle.componentwise_ratio(Cn, ii, jj, val, bound, K, np.float64)
        assert err <= max(err_n, 2.0 ** -53), (err, err_n)


def test_syrk_row_major_is_the_transposed_problem(blx, mode):
    N, K = 300, 200
    A = oracle.uniform((N, K), np.float64, 51)  # row-major N x K = column-major K x N
    C0 = oracle.uniform((N, N), np.float64, 52)
    Crm = C0.copy(order="F")
    # row-major, upper, no-trans: C_rm = A_rm A_rm^T on the row-major upper triangle
    blx.cblas_dsyrk(101, 121, 111, N, K, 0.5, A.T.copy(order="F"), K, 2.0, Crm, N)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    Ccm = C0.copy(order="F")
    blx.cblas_dsyrk(102, 122, 112, N, K, 0.5, A.T.copy(order="F"), K, 2.0, Ccm, N)
    np.testing.assert_array_equal(Crm, Ccm)


def test_syrk_k0_and_alpha0_scale_only_the_triangle(blx, mode):
    N = 257
    A = np.full((N, 3), np.nan, order="F")  # alpha == 0 or K == 0: A is not read
    C0 = oracle.uniform((N, N), np.float64, 61)
    for K, al in ((0, 1.0), (3, 0.0)):
        C = C0.copy(order="F")
        blx.cblas_dsyrk(102, 122, 111, N, K, al, A, N, -2.0, C, N)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        m = oracle.tri_mask("L", N)
        np.testing.assert_array_equal(C[m], -2.0 * C0[m])
        np.testing.assert_array_equal(C[~m], C0[~m])


def test_dsyrk_device_entry_matches_host(blx, mode):
    torch = pytest.importorskip("torch")
    N, K = 640, 512
    A = oracle.uniform((N, K), np.float64, 71)
    C0 = oracle.uniform((N, N), np.float64, 72)
    Ch = C0.copy(order="F")
    blx.cblas_dsyrk(102, 121, 111, N, K, 1.5, A, N, 0.25, Ch, N)
    dA = torch.from_numpy(A.T.copy()).cuda(); dC = torch.from_numpy(C0.T.copy()).cuda()
    s = torch.cuda.Stream(); s.wait_stream(torch.cuda.current_stream())
    assert blx.dsyrk_device("U", "N", N, K, 1.5, dA, N, 0.25, dC, N, stream=s) == 0
    torch.cuda.synchronize()
    Cd = dC.cpu().numpy().T
    m = oracle.tri_mask("U", N)
    np.testing.assert_array_equal(Cd[~m], C0[~m])
    np.testing.assert_allclose(Cd[m], Ch[m], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("emulated", [False, True])
def test_dsyrk_out_of_core(blx, emulated):
    """A 64 MiB budget forces the tile cache: C tiles outside the triangle
    are skipped, diagonal tiles masked."""
    blx.set_hbm_budget(64 << 20)
    blx.set_tile(512)
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI if emulated else blx.MODE_NATIVE)
    try:
        N, K = 2400, 1700  # A (33 MB, also B) and C (46 MB) exceed the 64 MiB budget
        A = oracle.uniform((K, N), np.float64, 81)
        C0 = oracle.uniform((N, N), np.float64, 82)
        C = C0.copy(order="F")
        blx.cblas_dsyrk(102, 122, 112, N, K, 1.0, A, K, 0.5, C, N)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        st = blx.call_stats()
        assert st["tile"] == 512 and st["path"] == (2 if emulated else 1)
        m = oracle.tri_mask("L", N)
        np.testing.assert_array_equal(C[~m], C0[~m])
        rng = np.random.default_rng(6)
        ii = rng.integers(0, N, 4000); jj = rng.integers(0, N, 4000)
        keep = ii >= jj
        ii, jj = ii[keep], jj[keep]
        val, bound = oracle.dd_entries("T", "N", N, N, K, 1.0, A, K, A, K, 0.5, C0, N, ii, jj)
        ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float64)
        assert ratio <= 1.0
    finally:
        blx.set_hbm_budget(0)
        blx.set_tile(0)
        blx.set_dgemm_mode(prev)


def test_syrk_through_the_serving_loop(blx):
    blx.serve_start(0, 0, 4)
    try:
        N, K = 900, 700
        A = oracle.uniform((N, K), np.float64, 91)
        C0 = oracle.uniform((N, N), np.float64, 92)
        C = C0.copy(order="F")
        blx.cblas_dsyrk(102, 121, 111, N, K, 1.0, A, N, 1.0, C, N)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    finally:
        blx.serve_stop()
    m = oracle.tri_mask("U", N)
    np.testing.assert_array_equal(C[~m], C0[~m])
    want = oracle.syrk("U", "N", N, K, 1.0, A, N, 1.0, C0.copy(order="F"), N)
    np.testing.assert_allclose(C[m], want[m], rtol=1e-11, atol=1e-11)
