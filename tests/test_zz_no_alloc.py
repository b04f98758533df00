"""GPU test of blasx_dgemm_device_noalloc, the DGEMM entry point that
allocates no memory (for callers whose device memory belongs to another
allocator, or that cannot afford cudaMalloc's synchronisation).

It is called through the C ABI and compared with blasx_dgemm_device (the
existing device-resident entry point, here on the same emulated path) on two
calls in a row of different shapes, so the second call runs on scratch that
still holds the first call's contents. The file is named to be collected
last; it passes alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _device(x, torch):
    # column-major numpy array -> device buffer with the same memory layout
    return torch.from_numpy(np.ascontiguousarray(x.T)).cuda()


def test_noalloc_matches_device_entry_on_two_calls(blx):
    torch = pytest.importorskip("torch")
    L = blx.lib()
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI)
    try:
        stream = torch.cuda.Stream()
        for (M, N, K, ta, tb, seed) in [(700, 513, 1000, "N", "T", 1), (1024, 1024, 1024, "T", "N", 5)]:
            ra, ca = oracle.shape_of_op(ta, M, K)
            rb, cb = oracle.shape_of_op(tb, K, N)
            A = oracle.uniform((ra, ca), np.float64, seed)
            B = oracle.uniform((rb, cb), np.float64, seed + 1)
            C0 = oracle.uniform((M, N), np.float64, seed + 2)
            dA, dB = _device(A, torch), _device(B, torch)
            d_ref, d_new = _device(C0, torch), _device(C0, torch)
            stream.wait_stream(torch.cuda.current_stream())
            st = blx.gemm_device(ta, tb, M, N, K, 1.5, dA, ra, dB, rb, -0.25, d_ref, M, stream=stream)
            assert st == blx.BLASX_OK, blx.last_error()
            st = L.blasx_dgemm_device_noalloc(blx.TRANS[ta], blx.TRANS[tb], M, N, K, 1.5, dA.data_ptr(), ra,
                                              dB.data_ptr(), rb, -0.25, d_new.data_ptr(), M, stream.cuda_stream)
            assert st == blx.BLASX_OK, blx.last_error()
            torch.cuda.synchronize()
            c_ref = d_ref.cpu().numpy().T
            c_new = d_new.cpu().numpy().T
            # tolerance of the parity tests: the componentwise bound (K+2) u (|alpha||A||B| + |beta||C0|)
            opA = A if ta == "N" else A.T
            opB = B if tb == "N" else B.T
            bound = 1.5 * (np.abs(opA) @ np.abs(opB)) + 0.25 * np.abs(C0)
            gamma = (K + 2) * 2.0 ** -53
            assert np.all(np.abs(c_new - c_ref) <= gamma * bound)
            rng = np.random.default_rng(seed)
            ii = rng.integers(0, M, 2000); jj = rng.integers(0, N, 2000)
            val, bnd = oracle.dd_entries(ta, tb, M, N, K, 1.5, A, ra, B, rb, -0.25, C0, M, ii, jj)
            ratio, _ = oracle.componentwise_ratio(c_new, ii, jj, val, bnd, K, np.float64)
            assert ratio <= 1.0
    finally:
        blx.set_dgemm_mode(prev)


def _dominant(shape, seed):
    """Column-major matrix whose every row and column is dominated by one
    entry of magnitude about 1 (the rest ~2^-30): the widest spread the
    modulus decision measures, so that no modulus count reaches FP64 accuracy
    and auto mode takes the native fallback on the device."""
    rng = np.random.default_rng(seed)
    x = oracle.uniform(shape, np.float64, seed) * 2.0 ** -30
    r, c = shape
    perm = rng.permutation(max(r, c))
    for t in range(max(r, c)):
        x[t % r, perm[t] % c] = rng.uniform(0.5, 1.0) * (1 if rng.random() < 0.5 else -1)
    return x


def test_noalloc_native_fallback_after_an_emulated_call(blx):
    """Auto mode, wide exponent spread: the decision left in the shared
    scratch by an emulated call is replaced, the device picks the native
    kernel, and the result equals the native kernel's bit for bit (the
    existing entry point sends this size to the native kernel)."""
    torch = pytest.importorskip("torch")
    L = blx.lib()
    prev = blx.set_dgemm_mode(blx.MODE_AUTO)
    try:
        stream = torch.cuda.Stream()
        M, N, K = 640, 384, 1000
        # an emulated call first (uniform operands), so the scratch holds a non-zero decision
        A0 = oracle.uniform((M, K), np.float64, 21)
        B0 = oracle.uniform((K, N), np.float64, 22)
        dA0, dB0 = _device(A0, torch), _device(B0, torch)
        dC0 = torch.zeros((N, M), dtype=torch.float64, device="cuda")
        stream.wait_stream(torch.cuda.current_stream())
        st = L.blasx_dgemm_device_noalloc(111, 111, M, N, K, 1.0, dA0.data_ptr(), M, dB0.data_ptr(), K, 0.0,
                                          dC0.data_ptr(), M, stream.cuda_stream)
        assert st == blx.BLASX_OK, blx.last_error()
        assert L.blasx_dgemm_device_noalloc_status(stream.cuda_stream) == blx.BLASX_OK
        # then the wide-spread call
        A = _dominant((M, K), 23)
        B = _dominant((K, N), 24)
        C0 = oracle.uniform((M, N), np.float64, 25)
        dA, dB = _device(A, torch), _device(B, torch)
        d_ref, d_new = _device(C0, torch), _device(C0, torch)
        stream.wait_stream(torch.cuda.current_stream())
        st = blx.gemm_device("N", "N", M, N, K, 1.25, dA, M, dB, K, 0.5, d_ref, M, stream=stream)
        assert st == blx.BLASX_OK, blx.last_error()
        st = L.blasx_dgemm_device_noalloc(111, 111, M, N, K, 1.25, dA.data_ptr(), M, dB.data_ptr(), K, 0.5,
                                          d_new.data_ptr(), M, stream.cuda_stream)
        assert st == blx.BLASX_OK, blx.last_error()
        assert L.blasx_dgemm_device_noalloc_status(stream.cuda_stream) == blx.BLASX_OK
        torch.cuda.synchronize()
        c_ref = d_ref.cpu().numpy().T
        c_new = d_new.cpu().numpy().T
        assert np.array_equal(c_new, c_ref)  # the same native kernel on the same operands
        rng = np.random.default_rng(3)
        ii = rng.integers(0, M, 2000); jj = rng.integers(0, N, 2000)
        val, bnd = oracle.dd_entries("N", "N", M, N, K, 1.25, A, M, B, K, 0.5, C0, M, ii, jj)
        ratio, _ = oracle.componentwise_ratio(c_new, ii, jj, val, bnd, K, np.float64)
        assert ratio <= 1.0
    finally:
        blx.set_dgemm_mode(prev)


def test_noalloc_follows_native_mode(blx):
    """Native mode: the FP64 kernel runs, as for blasx_dgemm_device."""
    torch = pytest.importorskip("torch")
    L = blx.lib()
    prev = blx.set_dgemm_mode(blx.MODE_NATIVE)
    try:
        M, N, K = 300, 200, 700
        A = oracle.uniform((K, M), np.float64, 31)
        B = oracle.uniform((N, K), np.float64, 32)
        C0 = oracle.uniform((M, N), np.float64, 33)
        dA, dB = _device(A, torch), _device(B, torch)
        d_ref, d_new = _device(C0, torch), _device(C0, torch)
        torch.cuda.synchronize()
        st = blx.gemm_device("T", "T", M, N, K, -0.75, dA, K, dB, N, 2.0, d_ref, M)
        assert st == blx.BLASX_OK, blx.last_error()
        st = L.blasx_dgemm_device_noalloc(112, 112, M, N, K, -0.75, dA.data_ptr(), K, dB.data_ptr(), N, 2.0,
                                          d_new.data_ptr(), M, None)
        assert st == blx.BLASX_OK, blx.last_error()
        assert L.blasx_dgemm_device_noalloc_status(None) == blx.BLASX_OK
        torch.cuda.synchronize()
        assert torch.equal(d_new, d_ref)
    finally:
        blx.set_dgemm_mode(prev)


def test_noalloc_reports_a_device_timeout(blx):
    """A bounded wait of the residue GEMM that runs out (test hook: one stage
    of CTA 0 is never loaded, every wait limited to about 1 ms) is reported by
    the status query, and the next call, hook disarmed, is correct."""
    torch = pytest.importorskip("torch")
    L = blx.lib()
    prev = blx.set_dgemm_mode(blx.MODE_OZAKI)
    try:
        M, N, K = 700, 513, 1000
        A = oracle.uniform((M, K), np.float64, 41)
        B = oracle.uniform((K, N), np.float64, 42)
        C0 = oracle.uniform((M, N), np.float64, 43)
        dA, dB = _device(A, torch), _device(B, torch)
        d_ref = _device(C0, torch)
        torch.cuda.synchronize()
        assert blx.gemm_device("N", "N", M, N, K, 1.5, dA, M, dB, K, -0.25, d_ref, M) == blx.BLASX_OK
        blx.test_stall_residue_gemm(1, 2_000_000)
        d_new = _device(C0, torch)
        torch.cuda.synchronize()
        st = L.blasx_dgemm_device_noalloc(111, 111, M, N, K, 1.5, dA.data_ptr(), M, dB.data_ptr(), K, -0.25,
                                          d_new.data_ptr(), M, None)
        assert st == blx.BLASX_OK, blx.last_error()
        assert L.blasx_dgemm_device_noalloc_status(None) == blx.BLASX_ERR_TIMEOUT
        d_new = _device(C0, torch)
        torch.cuda.synchronize()
        st = L.blasx_dgemm_device_noalloc(111, 111, M, N, K, 1.5, dA.data_ptr(), M, dB.data_ptr(), K, -0.25,
                                          d_new.data_ptr(), M, None)
        assert st == blx.BLASX_OK, blx.last_error()
        assert L.blasx_dgemm_device_noalloc_status(None) == blx.BLASX_OK
        torch.cuda.synchronize()
        assert torch.equal(d_new, d_ref)  # the same emulated pipeline on the same operands
    finally:
        blx.test_stall_residue_gemm(0, 1)
        blx.set_dgemm_mode(prev)


def test_noalloc_rejects_sizes_beyond_its_scratch(blx):
    torch = pytest.importorskip("torch")
    L = blx.lib()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    n = 2048  # needs more scratch than the fixed array holds; rejected before any device work
    st = L.blasx_dgemm_device_noalloc(111, 111, n, n, n, 1.0, buf.data_ptr(), n, buf.data_ptr(), n, 0.0,
                                      buf.data_ptr(), n, None)
    assert st == blx.BLASX_ERR_UNSUPPORTED
    assert "scratch" in blx.last_error()
    assert torch.all(buf == 0)
