"""CPU tests of the C ABI: the library loads, exports every declared symbol,
and reports illegal arguments exactly as the reference does (no GPU needed:
argument checking happens before any device work)."""
import ctypes
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_declared_symbols(blx):
    names = blx.declared_symbols()
    required = ["cblas_sgemm", "cblas_dgemm", "cblas_zgemm", "sgemm_", "dgemm_", "zgemm_", "xerbla_",
                "cblas_cgemm", "cgemm_"]
    for fam, types in (("syrk", "sdcz"), ("syr2k", "sdcz"), ("herk", "cz"), ("her2k", "cz"), ("symm", "sdcz"),
                       ("hemm", "cz"), ("trmm", "sdcz"), ("trsm", "sdcz")):
        required += [f"cblas_{t}{fam}" for t in types] + [f"{t}{fam}_" for t in types]
    missing_decl = [n for n in required if n not in names]
    assert not missing_decl, missing_decl
    out = subprocess.run(["nm", "-D", "--defined-only", blx.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if len(l.split()) >= 3}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = blx.lib()
    for n in names:
        assert getattr(L, n) is not None


def _capture(fn):
    libc = ctypes.CDLL(None)
    sys.stdout.flush()
    saved = os.dup(1)
    with tempfile.TemporaryFile(mode="w+b") as f:
        os.dup2(f.fileno(), 1)
        try:
            fn()
            libc.fflush(None)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        f.seek(0)
        return f.read().decode()


BAD = {1: dict(ta=999), 2: dict(tb=999), 3: dict(M=-1), 4: dict(N=-1), 5: dict(K=-1),
       8: dict(lda=2), 10: dict(ldb=2), 13: dict(ldc=2)}


@pytest.mark.parametrize("info", sorted(BAD))
@pytest.mark.parametrize("fn", ["cblas_dgemm", "cblas_sgemm"])
def test_xerbla_matches_reference(blx, golden, info, fn):
    want = [str(l) for l in golden["xerbla"] if str(l).startswith(f"{fn}|{info}|")][0].split("|", 2)[2]
    args = dict(ta=111, tb=111, M=4, N=4, K=4, lda=4, ldb=4, ldc=4)
    args.update(BAD[info])
    dt = np.float64 if fn == "cblas_dgemm" else np.float32
    A = np.zeros((4, 4), dt); B = np.zeros((4, 4), dt); C = np.ones((4, 4), dt, order="F")
    f = getattr(blx, fn)
    got = _capture(lambda: f(102, args["ta"], args["tb"], args["M"], args["N"], args["K"], 1.0, A,
                             args["lda"], B, args["ldb"], 0.0, C, args["ldc"]))
    assert got == want
    assert np.all(C == 1.0)
    assert blx.last_status() == blx.BLASX_ERR_ARG


@pytest.mark.parametrize("ta,tb", [("X", "N"), ("N", "Y"), ("X", "Y"), ("n", "c")])
def test_f77_trans_errors_match_reference(blx, golden, ta, tb):
    want = [str(l) for l in golden["xerbla"] if str(l).startswith(f"dgemm_{ta}{tb}|")][0].split("|", 2)[2]
    if want == "":
        pytest.skip("legal trans pair: runs a GEMM (covered by the GPU tests)")
    A = np.zeros((4, 4)); B = np.zeros((4, 4)); C = np.ones((4, 4), order="F")
    got = _capture(lambda: blx.dgemm_(ta, tb, 4, 4, 4, 1.0, A, 4, B, 4, 0.0, C, 4))
    assert got == want
    assert np.all(C == 1.0)


def test_zgemm_conjtrans_accepted_and_rowmajor_ld_rules(blx):
    # row-major: lda >= K for NoTrans A (M x K row-major); col-major would need lda >= M
    A = np.zeros((8, 3)); B = np.zeros((3, 2)); C = np.ones((8, 2))
    out = _capture(lambda: blx.cblas_dgemm(101, 111, 111, 8, 2, 3, 1.0, A, 2, B, 2, 0.0, C, 2))
    assert "parameter number  8" in out
    out = _capture(lambda: blx.cblas_dgemm(101, 111, 111, 8, 2, 3, 1.0, A, 3, B, 1, 0.0, C, 2))
    assert "parameter number 10" in out
    out = _capture(lambda: blx.cblas_dgemm(101, 111, 111, 8, 2, 3, 1.0, A, 3, B, 2, 0.0, C, 1))
    assert "parameter number 13" in out


def test_quick_return_needs_no_gpu(blx):
    # M == 0 or N == 0 returns before touching the device
    C = np.ones((4, 4), order="F")
    blx.cblas_dgemm(102, 111, 111, 0, 4, 4, 1.0, C, 4, C, 4, 0.0, C, 4)
    assert blx.last_status() == blx.BLASX_OK
    assert np.all(C == 1.0)


def test_no_gpu_fails_loudly():
    """Without a GPU the library reports BLASX_ERR_NODEVICE (no CPU fallback)."""
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np, blasx_b200 as b\n"
        "A=np.ones((4,4),order='F'); C=np.zeros((4,4),order='F')\n"
        "b.cblas_dgemm(102,111,111,4,4,4,1.0,A,4,A,4,0.0,C,4)\n"
        "print('STATUS', b.last_status(), float(C.sum()))\n" % ROOT)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=120)
    assert "STATUS 4 0.0" in r.stdout, (r.stdout, r.stderr)
    assert "no CUDA device" in r.stderr


def test_cgemm_reports_like_the_other_gemms(blx):
    # blas/cgemm.c:37-51 uses the same info numbering (first illegal argument wins)
    A = np.zeros((4, 4), np.complex64); C = np.ones((4, 4), np.complex64, order="F")
    out = _capture(lambda: blx.cblas_cgemm(102, 111, 111, 4, 4, 4, 1.0, A, 2, A, 4, 0.0, C, 4))
    assert out == " ** On entry to CGEMM  parameter number  8 had an illegal value\n"
    assert np.all(C == 1.0) and blx.last_status() == blx.BLASX_ERR_ARG
    out = _capture(lambda: blx.cgemm_("X", "N", 4, 4, 4, 1.0, A, 4, A, 4, 0.0, C, 4))
    assert "CGEMM  parameter number  1" in out
