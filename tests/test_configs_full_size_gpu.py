"""GPU parity at the benchmark configurations' full sizes.

* 4096^3 DGEMM NN, beta = 0.5, through cblas_dgemm on host arrays, native and
  auto precision: the whole C against OpenBLAS on the same arrays (both within
  the componentwise bound of the exact result, so within twice it of each
  other) and sampled entries against the double-double oracle.
* 8192^3 DGEMM NN, device-resident, entries U[-0.5,0.5] exp(phi g) for phi in
  {0, 1, 4}: emulated (auto) and native on the same inputs, both within the
  bound, the emulation no less accurate than the native kernel, and phi = 4
  taking the native fallback on the device.
* The ragged mixed-dtype calls at full size (sgemm TN and dgemm NT
  30001 x 17777 x 9999, zgemm CC 12001 x 8191 x 6007, alpha 1.5,
  beta -0.25) through cblas_?gemm, checked on sampled entries.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def sampled(C, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, ldc, dt, n=2000, seed=0):
    rng = np.random.default_rng(seed)
    ii = rng.integers(0, M, n); jj = rng.integers(0, N, n)
    val, bound = oracle.dd_entries(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C0, ldc, ii, jj)
    return oracle.componentwise_ratio(C, ii, jj, val, bound, K, dt)


@pytest.fixture
def mode_guard(blx):
    prev = blx.set_dgemm_mode(blx.MODE_AUTO)
    yield blx
    blx.set_dgemm_mode(prev)


@pytest.mark.parametrize("mode", ["native", "auto"])
def test_dgemm_4096_against_openblas(mode_guard, mode):
    blx = mode_guard
    n = 4096
    A = oracle.uniform((n, n), np.float64, 101)
    B = oracle.uniform((n, n), np.float64, 102)
    C0 = oracle.uniform((n, n), np.float64, 103)
    blx.set_dgemm_mode(blx.MODE_NATIVE if mode == "native" else blx.MODE_AUTO)
    C = C0.copy(order="F")
    blx.cblas_dgemm(102, 111, 111, n, n, n, 1.0, A, n, B, n, 0.5, C, n)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    assert blx.call_stats()["path"] == (1 if mode == "native" else 2)
    ob = oracle.OpenBLAS()
    Cob = C0.copy(order="F")
    ob.gemm("N", "N", n, n, n, 1.0, A, n, B, n, 0.5, Cob, n)
    absab = np.zeros((n, n), order="F")
    ob.gemm("N", "N", n, n, n, 1.0, np.abs(A), n, np.abs(B), n, 0.0, absab, n)
    gamma = (n + 2) * 2.0 ** -53
    bound = gamma * (absab + 0.5 * np.abs(C0))
    assert np.all(np.abs(C - Cob) <= 2.0 * bound)
    ratio, _ = sampled(C, "N", "N", n, n, n, 1.0, A, n, B, n, 0.5, C0, n, np.float64)
    assert ratio <= 1.0


@pytest.mark.parametrize("phi", [0.0, 1.0, 4.0])
def test_dgemm_8192_emulated_vs_native(mode_guard, phi):
    blx = mode_guard
    torch = pytest.importorskip("torch")
    n = 8192
    A = oracle.spread((n, n), 201, phi)
    B = oracle.spread((n, n), 202, phi)
    C0 = oracle.uniform((n, n), np.float64, 203)
    # column-major host arrays -> device buffers with the same layout
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    errs = {}
    for mode in (blx.MODE_AUTO, blx.MODE_NATIVE):
        blx.set_dgemm_mode(mode)
        dC = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
        torch.cuda.synchronize()
        st = blx.gemm_device("N", "N", n, n, n, 1.0, dA, n, dB, n, 0.5, dC, n)
        assert st == blx.BLASX_OK, blx.last_error()
        torch.cuda.synchronize()
        stats = blx.call_stats()
        C = dC.cpu().numpy().T
        ratio, err = sampled(C, "N", "N", n, n, n, 1.0, A, n, B, n, 0.5, C0, n, np.float64)
        assert ratio <= 1.0, (mode, phi, ratio)
        errs[mode] = err
        if mode == blx.MODE_AUTO:
            if phi == 4.0:
                assert stats["path"] == 4 and stats["moduli"] == 0, stats  # native fallback on the device
            else:
                assert stats["path"] == 2 and stats["moduli"] >= 14, stats
        del dC
    assert errs[blx.MODE_AUTO] <= max(errs[blx.MODE_NATIVE], 2.0 ** -53), errs


@pytest.mark.parametrize("dtype,ta,tb,M,N,K", [
    (np.float32, "T", "N", 30001, 17777, 9999),
    (np.float64, "N", "T", 30001, 17777, 9999),
    (np.complex128, "C", "C", 12001, 8191, 6007),
])
def test_ragged_full_size(mode_guard, dtype, ta, tb, M, N, K):
    blx = mode_guard
    ra, ca = oracle.shape_of_op(ta, M, K)
    rb, cb = oracle.shape_of_op(tb, K, N)
    A = oracle.uniform((ra, ca), dtype, 301)
    B = oracle.uniform((rb, cb), dtype, 302)
    C0 = oracle.uniform((M, N), dtype, 303)
    alpha, beta = (1.5, -0.25) if dtype != np.complex128 else (1.5 + 0j, -0.25 + 0j)
    fn = {np.float32: blx.cblas_sgemm, np.float64: blx.cblas_dgemm, np.complex128: blx.cblas_zgemm}[dtype]
    C = C0.copy(order="F")
    fn(102, oracle.TRANS_OF[ta], oracle.TRANS_OF[tb], M, N, K, alpha, A, ra, B, rb, beta, C, M)
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    assert blx.call_stats()["path"] in (1, 2, 4)
    ratio, _ = sampled(C, ta, tb, M, N, K, alpha, A, ra, B, rb, beta, C0, M, dtype)
    assert ratio <= 1.0
