"""GPU tests of the emulated (Ozaki scheme II, INT8 tensor-core) path.

Every case runs through the C ABI with the precision mode forced to the
emulated path and is checked against the double-double oracle: within the
componentwise bound (K+2) u (|alpha||A||B| + |beta||C0|), and -- the accuracy
target of the emulation -- with a measured max normalised error no worse than
the native FP64 kernel's on the same inputs.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture
def ozaki(blx):
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI)
    yield blx
    blx.set_dgemm_mode(prev)


def run(blx, dt, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    fn = {np.float64: blx.cblas_dgemm, np.float32: blx.cblas_sgemm, np.complex128: blx.cblas_zgemm,
          np.complex64: blx.cblas_cgemm}[dt]
    fn(102, oracle.TRANS_OF[ta], oracle.TRANS_OF[tb], M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    return blx.call_stats()


def sampled_error(C, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, ldc, dt, n=3000, seed=0):
    rng = np.random.default_rng(seed)
    ii = rng.integers(0, M, n); jj = rng.integers(0, N, n)
    val, bound = oracle.dd_entries(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, ldc, ii, jj)
    return oracle.componentwise_ratio(C, ii, jj, val, bound, K, dt)


def make(dt, ta, tb, M, N, K, seed, phi=None):
    ra, ca = oracle.shape_of_op(ta, M, K)
    rb, cb = oracle.shape_of_op(tb, K, N)
    if phi is None:
        A = oracle.uniform((ra, ca), dt, seed)
        B = oracle.uniform((rb, cb), dt, seed + 1)
    else:
        A = oracle.spread((ra, ca), seed, phi)
        B = oracle.spread((rb, cb), seed + 1, phi)
    C0 = oracle.uniform((M, N), dt, seed + 2)
    return A, ra, B, rb, C0


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("shape", [(300, 200, 170), (1000, 513, 777), (129, 1, 300), (1, 257, 64)])
def test_dgemm_emulated_vs_oracle(ozaki, blx, ta, tb, shape):
    M, N, K = shape
    A, lda, B, ldb, C0 = make(np.float64, ta, tb, M, N, K, 31)
    C = C0.copy(order="F")
    st = run(blx, np.float64, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C, M)
    assert st["path"] == 2 and st["moduli"] >= 12, st
    ratio, err = sampled_error(C, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C0, M, np.float64)
    assert ratio <= 1.0
    # native on the same inputs: the emulation must be at least as accurate
    blx.set_dgemm_mode(blx.MODE_NATIVE)
    Cn = C0.copy(order="F")
    run(blx, np.float64, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, Cn, M)
    blx.set_dgemm_mode(blx.MODE_OZAKI)
    _, err_n = sampled_error(Cn, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C0, M, np.float64)
    assert err <= max(err_n, 2.0 ** -53), (err, err_n)


def test_integer_inputs_are_exact(ozaki, blx):
    # small-integer operands: every product and sum is exact in FP64, so the
    # emulated result must equal the exact integer result bit for bit
    rng = np.random.default_rng(5)
    M, N, K = 517, 263, 1031
    A = np.asfortranarray(rng.integers(-64, 64, (M, K)).astype(np.float64))
    B = np.asfortranarray(rng.integers(-64, 64, (K, N)).astype(np.float64))
    C = np.zeros((M, N), order="F")
    run(blx, np.float64, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    want = (A.astype(np.int64) @ B.astype(np.int64)).astype(np.float64)
    np.testing.assert_array_equal(C, want)


@pytest.mark.parametrize("phi", [0.0, 1.0])
def test_spread_inputs_at_least_native_accuracy(ozaki, blx, phi):
    M = N = K = 1024
    A = oracle.spread((M, K), 41, phi); B = oracle.spread((K, N), 42, phi)
    C0 = np.zeros((M, N), order="F")
    C = C0.copy(order="F")
    st = run(blx, np.float64, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    assert st["path"] == 2
    ratio, err = sampled_error(C, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, None, M, np.float64)
    blx.set_dgemm_mode(blx.MODE_NATIVE)
    Cn = C0.copy(order="F")
    run(blx, np.float64, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, Cn, M)
    blx.set_dgemm_mode(blx.MODE_OZAKI)
    _, err_n = sampled_error(Cn, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, None, M, np.float64)
    assert ratio <= 1.0
    assert err <= err_n, (st["moduli"], err, err_n)


def test_auto_mode_falls_back_to_native_for_wide_spread(blx):
    prev = blx.set_dgemm_mode(blx.MODE_AUTO)
    try:
        M = N = K = 2048  # large enough for auto mode to pick the emulated path
        A = oracle.spread((M, K), 51, 4.0); B = oracle.spread((K, N), 52, 4.0)
        C = np.zeros((M, N), order="F")
        st = run(blx, np.float64, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, C, M)
        assert st["path"] == 4 and st["moduli"] == 0, st
        ratio, _ = sampled_error(C, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, None, M, np.float64)
        assert ratio <= 1.0
        # uniform data of the same size takes the emulated path in auto mode
        A = oracle.spread((M, K), 53, 0.0); B = oracle.spread((K, N), 54, 0.0)
        st = run(blx, np.float64, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, C, M)
        assert st["path"] == 2 and st["moduli"] >= 12, st
    finally:
        blx.set_dgemm_mode(prev)


def test_nonfinite_inputs_take_native_path(ozaki, blx):
    M = N = K = 256
    A = oracle.uniform((M, K), np.float64, 61); B = oracle.uniform((K, N), np.float64, 62)
    A[3, 5] = np.inf
    B[7, 9] = np.nan
    C = np.zeros((M, N), order="F")
    st = run(blx, np.float64, "N", "N", M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    assert st["path"] == 4
    want = A @ B
    np.testing.assert_array_equal(np.isnan(C), np.isnan(want))
    np.testing.assert_array_equal(np.isinf(C), np.isinf(want))


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
def test_sgemm_emulated_vs_oracle(ozaki, blx, ta, tb):
    M, N, K = 700, 333, 901
    A, lda, B, ldb, C0 = make(np.float32, ta, tb, M, N, K, 71)
    C = C0.copy(order="F")
    st = run(blx, np.float32, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C, M)
    assert st["path"] == 2 and 6 <= st["moduli"] <= 12, st
    ratio, _ = sampled_error(C, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C0, M, np.float32)
    assert ratio <= 1.0


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "C"), ("T", "C"), ("C", "N")])
def test_cgemm_emulated_vs_oracle(ozaki, blx, ta, tb):
    """complex64 on the INT8 path: FP32 accuracy target (u = 2^-24), results
    at least as accurate as the native complex64 kernel."""
    M, N, K = 400, 300, 350
    A, lda, B, ldb, C0 = make(np.complex64, ta, tb, M, N, K, 85)
    C = C0.copy(order="F")
    alpha, beta = 1.5 - 0.5j, -0.25 + 0.75j
    st = run(blx, np.complex64, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, M)
    assert st["path"] == 2 and 6 <= st["moduli"] <= 12, st
    ratio, err = sampled_error(C, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, M, np.complex64)
    assert ratio <= 1.0
    blx.set_dgemm_mode(blx.MODE_NATIVE)
    Cn = C0.copy(order="F")
    run(blx, np.complex64, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, Cn, M)
    blx.set_dgemm_mode(blx.MODE_OZAKI)
    _, err_n = sampled_error(Cn, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, M, np.complex64)
    assert err <= max(err_n, 2.0 ** -24), (err, err_n)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "C"), ("T", "C"), ("C", "N")])
def test_zgemm_emulated_vs_oracle(ozaki, blx, ta, tb):
    M, N, K = 400, 300, 350
    A, lda, B, ldb, C0 = make(np.complex128, ta, tb, M, N, K, 81)
    C = C0.copy(order="F")
    alpha, beta = 1.5 - 0.5j, -0.25 + 0.75j
    st = run(blx, np.complex128, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, M)
    assert st["path"] == 2, st
    ratio, err = sampled_error(C, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, M, np.complex128)
    assert ratio <= 1.0
    blx.set_dgemm_mode(blx.MODE_NATIVE)
    Cn = C0.copy(order="F")
    run(blx, np.complex128, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, Cn, M)
    blx.set_dgemm_mode(blx.MODE_OZAKI)
    _, err_n = sampled_error(Cn, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, M, np.complex128)
    assert err <= max(err_n, 2.0 ** -53), (err, err_n)


def test_device_entry_emulated_matches_host(ozaki, blx):
    torch = pytest.importorskip("torch")
    M, N, K = 640, 384, 512
    A = oracle.uniform((M, K), np.float64, 91); B = oracle.uniform((K, N), np.float64, 92)
    C = oracle.uniform((M, N), np.float64, 93)
    Ch = C.copy(order="F")
    blx.cblas_dgemm(102, 111, 111, M, N, K, 1.25, A, M, B, K, -0.5, Ch, M)
    dA = torch.from_numpy(A.T.copy()).cuda(); dB = torch.from_numpy(B.T.copy()).cuda()
    dC = torch.from_numpy(C.T.copy()).cuda()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    st = blx.gemm_device("N", "N", M, N, K, 1.25, dA, M, dB, K, -0.5, dC, M, stream=s, dtype="d")
    assert st == 0
    torch.cuda.synchronize()
    # same inputs, same deterministic pipeline: bitwise equal
    np.testing.assert_array_equal(dC.cpu().numpy().T, Ch)


def test_device_entry_emulated_wide_c(ozaki, blx):
    """N above 65535: the reconstruction is launched in column chunks."""
    torch = pytest.importorskip("torch")
    M, N, K = 64, 70001, 96
    A = oracle.uniform((M, K), np.float64, 94); B = oracle.uniform((K, N), np.float64, 95)
    C0 = oracle.uniform((M, N), np.float64, 96)
    dA = torch.from_numpy(A.T.copy()).cuda(); dB = torch.from_numpy(B.T.copy()).cuda()
    dC = torch.from_numpy(C0.T.copy()).cuda()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    assert blx.gemm_device("N", "N", M, N, K, 0.75, dA, M, dB, K, 0.5, dC, M, stream=s, dtype="d") == 0
    torch.cuda.synchronize()
    st = blx.call_stats()
    assert st["path"] == 2 and st["moduli"] > 0
    C = dC.cpu().numpy().T
    rng = np.random.default_rng(4)
    ii = rng.integers(0, M, 3000); jj = np.concatenate([rng.integers(65535, N, 1500), rng.integers(0, N, 1500)])
    val, bound = oracle.dd_entries("N", "N", M, N, K, 0.75, A, M, B, K, 0.5, C0, M, ii, jj)
    ratio, _ = oracle.componentwise_ratio(C, ii, jj, val, bound, K, np.float64)
    assert ratio <= 1.0


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_host_emulated_k_blocks(ozaki, blx, ta, tb):
    """K >= 4096: the host pipeline copies and computes K in two blocks
    (summed in FP64); beta C0 is added per C panel at the end."""
    M, N, K = 700, 2100, 5000
    A, lda, B, ldb, C0 = make(np.float64, ta, tb, M, N, K, 61)
    C = C0.copy(order="F")
    st = run(blx, np.float64, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C, M)
    assert st["path"] == 2 and st["moduli"] >= 12, st
    assert st["h2d_bytes"] == 8.0 * (M * K + K * N + M * N)
    ratio, err = sampled_error(C, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C0, M, np.float64)
    assert ratio <= 1.0
    blx.set_dgemm_mode(blx.MODE_NATIVE)
    Cn = C0.copy(order="F")
    run(blx, np.float64, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, Cn, M)
    blx.set_dgemm_mode(blx.MODE_OZAKI)
    _, err_n = sampled_error(Cn, ta, tb, M, N, K, 1.5, A, lda, B, ldb, -0.25, C0, M, np.float64)
    assert err <= max(err_n, 2.0 ** -53), (err, err_n)


def test_host_emulated_k_blocks_zgemm_beta_zero(ozaki, blx):
    M, N, K = 600, 500, 4500
    A = oracle.uniform((K, M), np.complex128, 64)
    B = oracle.uniform((N, K), np.complex128, 65)
    C = np.full((M, N), np.nan, dtype=np.complex128, order="F")  # beta = 0: C never read
    st = run(blx, np.complex128, "C", "C", M, N, K, 1 - 0.5j, A, K, B, N, 0, C, M)
    assert st["path"] == 2 and st["h2d_bytes"] == 16.0 * (M * K + K * N)
    want = (1 - 0.5j) * (A.conj().T @ B.conj().T)
    np.testing.assert_allclose(C, want, rtol=1e-12, atol=1e-11)


def test_host_k_blocks_second_block_falls_back(blx):
    """The K-blocks decide separately: uniform first half (emulated), a wide
    exponent spread in the second half (native on the device)."""
    prev = blx.set_dgemm_mode(blx.MODE_AUTO)
    try:
        M, N, K = 2048, 2048, 8192
        A = oracle.uniform((M, K), np.float64, 71)
        B = oracle.uniform((K, N), np.float64, 72)
        A[:, K // 2:] = oracle.spread((M, K // 2), 73, 6.0)
        B[K // 2:, :] = oracle.spread((K // 2, N), 74, 6.0)
        C0 = oracle.uniform((M, N), np.float64, 75)
        C = C0.copy(order="F")
        st = run(blx, np.float64, "N", "N", M, N, K, 1.0, A, M, B, K, 0.5, C, M)
        assert st["path"] == 4 and st["moduli"] == 0, st  # the last block's decision
        ratio, _ = sampled_error(C, "N", "N", M, N, K, 1.0, A, M, B, K, 0.5, C0, M, np.float64)
        assert ratio <= 1.0
    finally:
        blx.set_dgemm_mode(prev)
