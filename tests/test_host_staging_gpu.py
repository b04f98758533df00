"""Pageable host operands staged through pinned bounce buffers: every host
pipeline (in-core native, in-core emulated in K-blocks, out-of-core tiles,
streamed TRSM / TRMM, a column longer than one bounce buffer) gives results
bit-identical to the same call with the operands registered for the call
and with operands the caller pinned, and reports how it copied them."""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COL = 102
NOTRANS, TRANS = 111, 112
LEFT, RIGHT = 141, 142
UPPER, LOWER = 121, 122
NONUNIT = 131


def pinned_copy(a):
    import torch
    tdt = {np.float64: torch.float64, np.float32: torch.float32, np.complex128: torch.complex128}[a.dtype.type]
    buf = torch.empty(a.size, dtype=tdt, pin_memory=True).numpy()
    out = buf.reshape(a.shape, order="F")
    out[...] = a
    return out, buf


@pytest.fixture
def settings(blx):
    yield blx
    blx.set_host_staging(True)
    blx.set_dgemm_mode(0)
    blx.set_hbm_budget(0)
    blx.set_tile(0)


def three_ways(blx, call, arrays, out_index):
    """Runs call(*arrays) staged, registered and caller-pinned; returns the
    three outputs (arrays[out_index] after each call) and host_copy modes."""
    outs, modes = [], []
    for way in ("staged", "registered", "pinned"):
        blx.set_host_staging(way != "registered")
        keep = []
        if way == "pinned":
            args = []
            for a in arrays:
                p, buf = pinned_copy(a)
                keep.append(buf)
                args.append(p)
        else:
            args = [a.copy(order="F") for a in arrays]
        call(*args)
        assert blx.last_status() == blx.BLASX_OK, blx.last_error()
        modes.append(blx.call_stats()["host_copy"])
        outs.append(np.array(args[out_index], copy=True))
    return outs, modes


def assert_identical(outs, modes):
    assert modes == [1, 2, 0], modes
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])


def gemm_case(rng, dt, M, N, K, ta, tb, pad=5):
    ra, ca = (M, K) if ta == NOTRANS else (K, M)
    rb, cb = (K, N) if tb == NOTRANS else (N, K)
    mk = (lambda r, c: rng.uniform(-1, 1, (r, c)) + 1j * rng.uniform(-1, 1, (r, c))) \
        if np.issubdtype(dt, np.complexfloating) else (lambda r, c: rng.uniform(-1, 1, (r, c)))
    A = np.asfortranarray(mk(ra + pad, ca).astype(dt))
    B = np.asfortranarray(mk(rb + pad, cb).astype(dt))
    C = np.asfortranarray(mk(M + pad, N).astype(dt))
    return A, B, C


@pytest.mark.parametrize("name,mode,M,N,K,ta,tb", [
    ("incore_native", 1, 3001, 2500, 2047, NOTRANS, TRANS),
    ("incore_emulated_kblocks", 2, 2048, 1536, 8192, TRANS, NOTRANS),
    ("incore_emulated", 2, 1800, 2100, 1500, NOTRANS, NOTRANS),
])
def test_dgemm_staged_equals_registered_and_pinned(settings, name, mode, M, N, K, ta, tb):
    blx = settings
    blx.set_dgemm_mode(mode)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    A, B, C = gemm_case(rng, np.float64, M, N, K, ta, tb)

    def call(A, B, C):
        blx.cblas_dgemm(COL, ta, tb, M, N, K, 0.75, A, A.shape[0], B, B.shape[0], -1.25, C, C.shape[0])

    outs, modes = three_ways(blx, call, [A, B, C], 2)
    assert_identical(outs, modes)
    # rows below M (the ld padding) are never written
    np.testing.assert_array_equal(outs[0][M:, :], C[M:, :])


@pytest.mark.parametrize("mode", [1, 2])
def test_out_of_core_staged_equals_registered_and_pinned(settings, mode):
    blx = settings
    blx.set_dgemm_mode(mode)
    blx.set_tile(512)
    blx.set_hbm_budget(48 << 20)
    rng = np.random.default_rng(7 + mode)
    M, N, K = 2300, 1900, 2100
    A, B, C = gemm_case(rng, np.float64, M, N, K, NOTRANS, NOTRANS)

    def call(A, B, C):
        blx.cblas_dgemm(COL, NOTRANS, NOTRANS, M, N, K, 1.0, A, A.shape[0], B, B.shape[0], 0.5, C, C.shape[0])

    outs, modes = three_ways(blx, call, [A, B, C], 2)
    assert blx.call_stats()["cache_misses"] > 0  # ran through the tile cache
    assert_identical(outs, modes)


def test_zgemm_staged_equals_registered_and_pinned(settings):
    blx = settings
    rng = np.random.default_rng(11)
    M, N, K = 1200, 900, 1000
    A, B, C = gemm_case(rng, np.complex128, M, N, K, NOTRANS, TRANS)

    def call(A, B, C):
        blx.cblas_zgemm(COL, NOTRANS, TRANS, M, N, K, 0.5 - 0.25j, A, A.shape[0], B, B.shape[0], 1.0 + 0.5j, C,
                        C.shape[0])

    outs, modes = three_ways(blx, call, [A, B, C], 2)
    assert_identical(outs, modes)


def test_column_longer_than_a_bounce_buffer(settings):
    # 4.3e6 rows x 8 bytes = 34.4 MB per column: each column is copied in
    # segments (a bounce buffer holds 32 MiB)
    blx = settings
    blx.set_dgemm_mode(1)
    rng = np.random.default_rng(5)
    M, N, K = 4_300_000, 3, 2
    A, B, C = gemm_case(rng, np.float64, M, N, K, NOTRANS, NOTRANS, pad=0)

    def call(A, B, C):
        blx.cblas_dgemm(COL, NOTRANS, NOTRANS, M, N, K, 1.0, A, M, B, K, 1.0, C, M)

    outs, modes = three_ways(blx, call, [A, B, C], 2)
    assert_identical(outs, modes)
    ref = A @ B + C
    np.testing.assert_allclose(outs[0], ref, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("kind", ["trsm", "trmm"])
@pytest.mark.parametrize("side", [LEFT, RIGHT])
def test_triangular_staged_equals_registered_and_pinned(settings, kind, side):
    # B is read and written back block by block (its parts are disjoint);
    # the triangle streams in strips
    blx = settings
    rng = np.random.default_rng(3 + side)
    M, N = 1700, 1300
    K = M if side == LEFT else N
    A = np.asfortranarray(np.tril(rng.uniform(-1, 1, (K + 3, K))) + K * np.eye(K + 3, K))
    B = np.asfortranarray(rng.uniform(-1, 1, (M + 2, N)))
    fn = blx.cblas_dtrsm if kind == "trsm" else blx.cblas_dtrmm

    def call(A, B):
        fn(COL, side, LOWER, NOTRANS, NONUNIT, M, N, 1.5, A, A.shape[0], B, B.shape[0])

    outs, modes = three_ways(blx, call, [A, B], 1)
    assert_identical(outs, modes)
