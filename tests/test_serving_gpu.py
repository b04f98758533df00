"""GPU tests of the serving loop: many host threads, continuous batching,
grouped launches, the operand cache and its identity rule, admission under a
small HBM budget. Every request's result in the concurrent mix is compared
with the same request run alone (serving stopped), and with the oracle."""
import threading

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

DT = [np.float64, np.float32, np.complex128]


def make_requests(n, seed, dmax=700):
    rng = np.random.default_rng(seed)
    reqs = []
    for t in range(n):
        dt = DT[rng.choice(3, p=[0.6, 0.3, 0.1])]
        M, N, K = (int(np.exp(rng.uniform(np.log(16), np.log(dmax)))) for _ in range(3))
        ta = "N" if dt == np.float32 and rng.random() < 0.5 else str(rng.choice(["N", "T"] + (["C"] if dt == np.complex128 else [])))
        tb = str(rng.choice(["N", "T"] + (["C"] if dt == np.complex128 else [])))
        ra, ca = oracle.shape_of_op(ta, M, K)
        rb, cb = oracle.shape_of_op(tb, K, N)
        A = oracle.uniform((ra, ca), dt, seed * 1000 + 3 * t)
        B = oracle.uniform((rb, cb), dt, seed * 1000 + 3 * t + 1)
        C0 = oracle.uniform((M, N), dt, seed * 1000 + 3 * t + 2)
        alpha, beta = (1.5, -0.25) if dt != np.complex128 else (1 - 0.5j, 0.25 + 0.5j)
        reqs.append(dict(dt=dt, ta=ta, tb=tb, M=M, N=N, K=K, A=A, ra=ra, B=B, rb=rb, C0=C0, alpha=alpha, beta=beta))
    return reqs


def run(blx, r):
    C = r["C0"].copy(order="F")
    fn = {np.float64: blx.cblas_dgemm, np.float32: blx.cblas_sgemm, np.complex128: blx.cblas_zgemm}[r["dt"]]
    fn(102, oracle.TRANS_OF[r["ta"]], oracle.TRANS_OF[r["tb"]], r["M"], r["N"], r["K"], r["alpha"], r["A"], r["ra"],
       r["B"], r["rb"], r["beta"], C, r["M"])
    assert blx.last_status() == blx.BLASX_OK, blx.last_error()
    return C


def bound(r):
    opA = r["A"] if r["ta"] == "N" else r["A"].T
    opB = r["B"] if r["tb"] == "N" else r["B"].T
    u = oracle.UNIT_ROUNDOFF[np.dtype(r["dt"]).type]
    g = (r["K"] + 2) * u * (2.0 if r["dt"] == np.complex128 else 1.0)
    return g * (abs(r["alpha"]) * (np.abs(opA).astype(np.float64) @ np.abs(opB).astype(np.float64))
                + abs(r["beta"]) * np.abs(r["C0"]).astype(np.float64))


@pytest.fixture
def serving(blx):
    yield blx
    blx.serve_stop()


def test_alone_equals_mix(serving):
    blx = serving
    reqs = make_requests(96, 1)
    alone = [run(blx, r) for r in reqs]  # serving stopped: one call at a time
    blx.serve_start(0, 0, 8)
    out = [None] * len(reqs)
    errs = []

    def worker(w):
        try:
            for i in range(w, len(reqs), 16):
                out[i] = run(blx, reqs[i])
        except Exception as e:  # pragma: no cover
            errs.append(e)

    th = [threading.Thread(target=worker, args=(w,)) for w in range(16)]
    [t.start() for t in th]
    [t.join() for t in th]
    assert not errs, errs
    st = blx.serve_stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["grouped_launches"] >= 1 and st["grouped_requests"] >= 2
    assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]
    for r, a, m in zip(reqs, alone, out):
        # the same deterministic kernels in both runs: equal within the stated bound
        assert np.all(np.abs(m - a) <= bound(r)), (r["M"], r["N"], r["K"], r["dt"])


def make_large_requests(seed):
    """Requests large enough for auto mode to emulate them (FP64 work >= 6e9
    with K >= 512, FP32 >= 3e8 with K >= 256, complex128 >= 2e9), in a mix
    with small native ones of every dtype."""
    rng = np.random.default_rng(seed)
    shapes = [(np.float64, 2048, 2048, 1536), (np.float64, 2304, 1792, 2048), (np.float64, 1800, 2100, 1700),
              (np.float32, 1024, 1024, 512), (np.float32, 1500, 900, 700), (np.complex128, 1280, 1280, 1280),
              (np.float64, 300, 200, 100), (np.float32, 200, 300, 150), (np.complex128, 100, 120, 90),
              (np.float64, 700, 500, 300)]
    reqs = []
    for t, (dt, M, N, K) in enumerate(shapes):
        ta = str(rng.choice(["N", "T"] + (["C"] if dt == np.complex128 else [])))
        tb = str(rng.choice(["N", "T"] + (["C"] if dt == np.complex128 else [])))
        ra, ca = oracle.shape_of_op(ta, M, K)
        rb, cb = oracle.shape_of_op(tb, K, N)
        A = oracle.uniform((ra, ca), dt, seed * 1000 + 3 * t)
        B = oracle.uniform((rb, cb), dt, seed * 1000 + 3 * t + 1)
        C0 = oracle.uniform((M, N), dt, seed * 1000 + 3 * t + 2)
        alpha, beta = (1.5, -0.25) if dt != np.complex128 else (1 - 0.5j, 0.25 + 0.5j)
        reqs.append(dict(dt=dt, ta=ta, tb=tb, M=M, N=N, K=K, A=A, ra=ra, B=B, rb=rb, C0=C0, alpha=alpha, beta=beta))
    return reqs


def test_alone_equals_mix_with_emulated_requests(serving):
    """Emulated FP64, FP32 and complex128 requests beside small native ones:
    each result in the concurrent mix equals the same request served alone
    bit for bit when it was emulated (exact integer products, per-request
    decision), and is within the bound of the unserved call's result."""
    blx = serving
    prev = blx.set_dgemm_mode(blx.MODE_AUTO)
    try:
        reqs = make_large_requests(3)
        unserved = [run(blx, r) for r in reqs]
        blx.serve_start(0, 0, 8)
        alone = []
        for r in reqs:
            alone.append(run(blx, r))
            if r["M"] >= 1000:  # large enough for auto mode: the executor runs it emulated
                assert blx.call_stats()["path"] == 2, (r["M"], r["N"], r["K"], r["dt"], blx.call_stats())
        out = [None] * len(reqs)
        errs = []

        def worker(w):
            try:
                for i in range(w, len(reqs), 10):
                    out[i] = run(blx, reqs[i])
            except Exception as e:  # pragma: no cover
                errs.append(e)

        for _ in range(2):
            th = [threading.Thread(target=worker, args=(w,)) for w in range(10)]
            [t.start() for t in th]
            [t.join() for t in th]
            assert not errs, errs
            for r, a, u, m in zip(reqs, alone, unserved, out):
                assert np.all(np.abs(m - u) <= 2 * bound(r)), (r["M"], r["N"], r["K"], r["dt"])
                if r["M"] >= 1000:  # emulated in both runs
                    assert np.array_equal(m, a), (r["M"], r["N"], r["K"], r["dt"])
        st = blx.serve_stats()
        assert st["failed"] == 0
    finally:
        blx.set_dgemm_mode(prev)


def test_operand_cache_hits_and_identity(serving):
    blx = serving
    blx.serve_start(0, 1 << 30, 4)
    M = N = K = 600
    A = oracle.uniform((M, K), np.float64, 5)
    B = oracle.uniform((K, N), np.float64, 6)
    C = np.zeros((M, N), order="F")
    for _ in range(3):
        blx.cblas_dgemm(102, 111, 111, M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    st = blx.serve_stats()
    assert st["cache_hits"] == 2 and st["cache_misses"] == 1
    np.testing.assert_allclose(C, A @ B, rtol=1e-12, atol=1e-12)
    # the host buffer changes: the fingerprint changes, the stale copy is not used
    B *= 2.0
    blx.cblas_dgemm(102, 111, 111, M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    np.testing.assert_allclose(C, A @ B, rtol=1e-12, atol=1e-12)
    # an in-place change of one element: the documented contract is invalidate()
    B[123, 321] += 1.0
    assert blx.serve_invalidate(B) >= 1
    blx.cblas_dgemm(102, 111, 111, M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    np.testing.assert_allclose(C, A @ B, rtol=1e-12, atol=1e-12)


def test_admission_under_small_budget(serving):
    blx = serving
    # room for about two of these requests at a time; all must still complete
    blx.serve_start(48 << 20, 8 << 20, 16)
    reqs = make_requests(24, 7, dmax=1500)
    out = [None] * len(reqs)

    def worker(w):
        for i in range(w, len(reqs), 8):
            out[i] = run(blx, reqs[i])

    th = [threading.Thread(target=worker, args=(w,)) for w in range(8)]
    [t.start() for t in th]
    [t.join() for t in th]
    st = blx.serve_stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for r, m in zip(reqs, out):
        opA = r["A"] if r["ta"] == "N" else (r["A"].T if r["ta"] == "T" else r["A"].conj().T)
        opB = r["B"] if r["tb"] == "N" else (r["B"].T if r["tb"] == "T" else r["B"].conj().T)
        want = r["alpha"] * (opA.astype(np.complex128) @ opB.astype(np.complex128)) + r["beta"] * r["C0"]
        assert np.all(np.abs(m - want) <= 4 * bound(r) + 1e-300)
