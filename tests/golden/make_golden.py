"""Generate the golden GEMM fixtures from the reference library itself.

The reference (linnanwang/BLASX) is compiled from its own, unmodified sources
into ``oracle/_ref/libblasx_ref.so`` by ``oracle/Makefile`` (a one-header
include shim only). Every call made here keeps all dimensions <= 500, so the
reference dispatches it to its CPU BLAS path (blas/dgemm.c:61-75,
blas/zgemm.c:59-75): these are the reference's own outputs for the path.

Also recorded: the exact xerbla_ lines the reference prints for each illegal
argument (blas/dgemm.c:46-57, blas/error.c:5-8) and for the F77 wrappers
(blas/dgemm.c:131-154).

SYRK and SYR2K: the reference runs cblas_?syrk / cblas_?syr2k on its CPU BLAS
for every size (blas/dsyrk.c:36-39, blas/dsyr2k.c); their outputs and the
reference's xerbla_ lines for each illegal argument (blas/dsyrk.c:27-37,
blas/dsyr2k.c:43-52, the F77 wrappers blas/dsyrk.c:80-101) are recorded too.

The reference's CPU BLAS is multithreaded, so a run on another machine may
differ from the recorded outputs in the last bits; the tests compare within
the componentwise bound, and a regeneration should keep the recorded entries
and add only new ones.

Run in a container that has the reference tree:  python tests/golden/make_golden.py
"""
import ctypes
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gemm_golden.npz")

SHAPES = [(1, 1, 1), (7, 5, 3), (33, 17, 65), (5, 129, 2), (64, 64, 64), (130, 70, 45)]
BIG = {(64, 64, 64), (130, 70, 45)}  # only NN / first scalar pair at these sizes
SCALARS = [(1.0, 0.0), (1.5, -0.25), (0.0, 0.5), (-0.25, 1.0)]
ZSCALARS = [((1.0, 0.0), (0.0, 0.0)), ((1.5, -0.5), (-0.25, 0.75)), ((0.0, 0.0), (0.5, -1.0))]


def capture_stdout(fn):
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


def main():
    ref = oracle.Reference()
    rec = {}
    n = 0
    # complex64 last, so that the earlier cases keep their numbering (and seeds)
    dtypes = [("d", np.float64, "NT"), ("s", np.float32, "NT"), ("z", np.complex128, "NTC"),
              ("c", np.complex64, "NTC")]
    for tag, dt, transes in dtypes:
        for (M, N, K) in SHAPES:
            scal = ZSCALARS if tag in "zc" else SCALARS
            for ta in transes:
                for tb in transes:
                    for si, (al, be) in enumerate(scal):
                        # all trans combos on the first scalar pair; all pairs on NN/TN
                        if si > 0 and not (tb == "N"):
                            continue
                        if (M, N, K) in BIG and not (ta == "N" and tb == "N" and si <= 1):
                            continue
                        if tag in "zc":
                            al = complex(*al); be = complex(*be)
                        seed = 1000 + n
                        ra, ca = oracle.shape_of_op(ta, M, K)
                        rb, cb = oracle.shape_of_op(tb, K, N)
                        lda, ldb, ldc = ra + (n % 3), rb + (n % 2), M + (n % 4)
                        A = oracle.uniform((lda, ca), dt, seed)
                        B = oracle.uniform((ldb, cb), dt, seed + 1)
                        C = oracle.uniform((ldc, N), dt, seed + 2)
                        C0 = C.copy(order="F")
                        ref.gemm(ta, tb, M, N, K, al, A, lda, B, ldb, be, C, ldc)
                        key = f"{tag}_{n}"
                        rec[key + "_meta"] = np.array([M, N, K, lda, ldb, ldc, ord(ta), ord(tb)], dtype=np.int64)
                        rec[key + "_scal"] = np.array([al, be], dtype=np.complex128)
                        # inputs are regenerated from the seed; a checksum guards the generator
                        rec[key + "_seed"] = np.array([seed], dtype=np.int64)
                        rec[key + "_sum"] = np.array([np.sum(A), np.sum(B), np.sum(C0)], dtype=np.complex128)
                        rec[key + "_C"] = C
                        n += 1
    # degenerate cases: K = 0 (C <- beta C), beta = 0 with NaN in C, alpha = 0 with NaN in A/B
    for case, (M, N, K, al, be, nanA, nanC) in enumerate(
            [(9, 7, 0, 1.5, -0.25, False, False), (9, 7, 5, 1.5, 0.0, False, True),
             (9, 7, 5, 0.0, 0.5, True, False)]):
        A = oracle.uniform((M, max(K, 1)), np.float64, 77 + case)
        B = oracle.uniform((max(K, 1), N), np.float64, 88 + case)
        C = oracle.uniform((M, N), np.float64, 99 + case)
        if nanA:
            A[:] = np.nan; B[:] = np.nan
        if nanC:
            C[:] = np.nan
        C0 = C.copy(order="F")
        ref.gemm("N", "N", M, N, K, al, A, M, B, max(K, 1), be, C, M)
        key = f"edge_{case}"
        rec[key + "_meta"] = np.array([M, N, K, M, max(K, 1), M, ord("N"), ord("N")], dtype=np.int64)
        rec[key + "_scal"] = np.array([al, be], dtype=np.complex128)
        rec[key + "_A"] = A; rec[key + "_B"] = B; rec[key + "_C0"] = C0; rec[key + "_C"] = C
    # SYRK / SYR2K outputs of the reference (its CPU BLAS path)
    I, D, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    L = ref.L
    L.cblas_dsyrk.argtypes = [I] * 5 + [D, P, I, D, P, I]
    L.cblas_ssyrk.argtypes = [I] * 5 + [ctypes.c_float, P, I, ctypes.c_float, P, I]
    L.cblas_zsyrk.argtypes = [I] * 5 + [P, P, I, P, P, I]
    L.cblas_dsyr2k.argtypes = [I] * 5 + [D, P, I, P, I, D, P, I]
    ns = 0
    for tag, dt in (("d", np.float64), ("s", np.float32), ("z", np.complex128)):
        for (N, K) in [(1, 1), (7, 3), (33, 65), (64, 17)]:
            for uplo in (121, 122):
                for trans in (111, 112):
                    seed = 5000 + ns
                    ra, ca = (N, K) if trans == 111 else (K, N)
                    lda, ldc = ra + (ns % 2), N + (ns % 3)
                    A = oracle.uniform((lda, ca), dt, seed)
                    C = oracle.uniform((ldc, N), dt, seed + 1)
                    C0 = C.copy(order="F")
                    al, be = (1.5, -0.25) if tag != "z" else (complex(1.5, -0.5), complex(-0.25, 0.75))
                    if tag == "d":
                        L.cblas_dsyrk(102, uplo, trans, N, K, al, A.ctypes.data, lda, be, C.ctypes.data, ldc)
                    elif tag == "s":
                        L.cblas_ssyrk(102, uplo, trans, N, K, al, A.ctypes.data, lda, be, C.ctypes.data, ldc)
                    else:
                        pa = np.array([al.real, al.imag]); pb = np.array([be.real, be.imag])
                        L.cblas_zsyrk(102, uplo, trans, N, K, pa.ctypes.data, A.ctypes.data, lda, pb.ctypes.data,
                                      C.ctypes.data, ldc)
                    key = f"syrk_{tag}_{ns}"
                    rec[key + "_meta"] = np.array([N, K, uplo, trans, lda, ldc, seed], dtype=np.int64)
                    rec[key + "_scal"] = np.array([al, be], dtype=np.complex128)
                    rec[key + "_sum"] = np.array([np.sum(A), np.sum(C0)], dtype=np.complex128)
                    rec[key + "_C"] = C
                    ns += 1
    for (N, K) in [(7, 3), (33, 65)]:
        for uplo in (121, 122):
            for trans in (111, 112):
                seed = 6000 + ns
                ra, ca = (N, K) if trans == 111 else (K, N)
                A = oracle.uniform((ra, ca), np.float64, seed)
                B = oracle.uniform((ra, ca), np.float64, seed + 1)
                C = oracle.uniform((N, N), np.float64, seed + 2)
                C0 = C.copy(order="F")
                L.cblas_dsyr2k(102, uplo, trans, N, K, 1.5, A.ctypes.data, ra, B.ctypes.data, ra, -0.25,
                               C.ctypes.data, N)
                key = f"syr2k_d_{ns}"
                rec[key + "_meta"] = np.array([N, K, uplo, trans, ra, N, seed], dtype=np.int64)
                rec[key + "_sum"] = np.array([np.sum(A), np.sum(B), np.sum(C0)], dtype=np.complex128)
                rec[key + "_C"] = C
                ns += 1
    # xerbla lines for every info code of cblas_dgemm and the F77 wrapper
    A = np.zeros((4, 4)); B = np.zeros((4, 4)); C = np.ones((4, 4), order="F")
    bad = {
        1: dict(ta=999), 2: dict(tb=999), 3: dict(M=-1), 4: dict(N=-1), 5: dict(K=-1),
        8: dict(lda=2), 10: dict(ldb=2), 13: dict(ldc=2),
    }
    lines = []
    for info, kw in bad.items():
        args = dict(ta=111, tb=111, M=4, N=4, K=4, lda=4, ldb=4, ldc=4)
        args.update(kw)
        out = capture_stdout(lambda: ref.L.cblas_dgemm(102, args["ta"], args["tb"], args["M"], args["N"], args["K"],
                                                       1.0, A.ctypes.data, args["lda"], B.ctypes.data, args["ldb"],
                                                       0.0, C.ctypes.data, args["ldc"]))
        lines.append(f"cblas_dgemm|{info}|{out}")
        out = capture_stdout(lambda: ref.L.cblas_sgemm(102, args["ta"], args["tb"], args["M"], args["N"], args["K"],
                                                       1.0, A.astype(np.float32).ctypes.data, args["lda"],
                                                       B.astype(np.float32).ctypes.data, args["ldb"], 0.0,
                                                       C.astype(np.float32).ctypes.data, args["ldc"]))
        lines.append(f"cblas_sgemm|{info}|{out}")
    assert np.all(C == 1.0), "C must be untouched on argument errors"
    for ta, tb in [(b"X", b"N"), (b"N", b"Y"), (b"X", b"Y"), (b"n", b"c")]:
        m = ctypes.c_int(4); k = ctypes.c_int(4); ld = ctypes.c_int(4)
        al = ctypes.c_double(1.0); be = ctypes.c_double(0.0)
        Cz = np.zeros((4, 4), order="F")
        tab = ctypes.c_char(ta); tbb = ctypes.c_char(tb)
        out = capture_stdout(lambda: ref.L.dgemm_(ctypes.byref(tab), ctypes.byref(tbb), ctypes.byref(m),
                                                  ctypes.byref(m), ctypes.byref(k), ctypes.byref(al),
                                                  A.ctypes.data, ctypes.byref(ld), B.ctypes.data,
                                                  ctypes.byref(ld), ctypes.byref(be), Cz.ctypes.data,
                                                  ctypes.byref(ld)))
        lines.append(f"dgemm_{ta.decode()}{tb.decode()}|-|{out}")
    # SYRK / SYR2K argument errors
    Cs = np.ones((4, 4), order="F")
    for info, kw in {1: dict(uplo=999), 2: dict(trans=999), 3: dict(N=-1), 4: dict(K=-1), 7: dict(lda=2),
                     10: dict(ldc=2)}.items():
        a = dict(uplo=121, trans=111, N=4, K=4, lda=4, ldc=4)
        a.update(kw)
        out = capture_stdout(lambda: L.cblas_dsyrk(102, a["uplo"], a["trans"], a["N"], a["K"], 1.0, A.ctypes.data,
                                                   a["lda"], 0.0, Cs.ctypes.data, a["ldc"]))
        lines.append(f"cblas_dsyrk|{info}|{out}")
    for info, kw in {7: dict(lda=2), 9: dict(ldb=2), 12: dict(ldc=2)}.items():
        a = dict(lda=4, ldb=4, ldc=4)
        a.update(kw)
        out = capture_stdout(lambda: L.cblas_dsyr2k(102, 121, 111, 4, 4, 1.0, A.ctypes.data, a["lda"], B.ctypes.data,
                                                    a["ldb"], 0.0, Cs.ctypes.data, a["ldc"]))
        lines.append(f"cblas_dsyr2k|{info}|{out}")
    L.dsyrk_.argtypes = [P] * 10
    for up, tr in [(b"X", b"N"), (b"U", b"Q"), (b"X", b"Q")]:
        nn = ctypes.c_int(4); ld = ctypes.c_int(4)
        al = ctypes.c_double(1.0); be = ctypes.c_double(0.0)
        cu = ctypes.c_char(up); ct = ctypes.c_char(tr)
        out = capture_stdout(lambda: L.dsyrk_(ctypes.byref(cu), ctypes.byref(ct), ctypes.byref(nn), ctypes.byref(nn),
                                              ctypes.byref(al), A.ctypes.data, ctypes.byref(ld), ctypes.byref(be),
                                              Cs.ctypes.data, ctypes.byref(ld)))
        lines.append(f"dsyrk_{up.decode()}{tr.decode()}|-|{out}")
    assert np.all(Cs == 1.0), "C must be untouched on argument errors"
    rec["xerbla"] = np.array(lines)
    np.savez_compressed(OUT, **rec)
    print(f"wrote {OUT}: {n} GEMM cases + 3 edge cases + {ns} SYRK/SYR2K cases + {len(lines)} xerbla lines")


if __name__ == "__main__":
    main()
