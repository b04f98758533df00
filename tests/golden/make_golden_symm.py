"""Generate the SYMM / HEMM / TRMM / TRSM and HERK / HER2K / CSYRK / CSYR2K
golden fixtures from the reference library.

The reference (linnanwang/BLASX) is compiled from its own, unmodified sources
into ``oracle/_ref/libblasx_ref.so`` by ``oracle/Makefile``. Its cblas_?symm,
cblas_?hemm, cblas_?trmm and cblas_?trsm send every call to its CPU BLAS
(blas/dsymm.c:44-57, blas/zhemm.c, blas/dtrmm.c:43-60, blas/dtrsm.c:44-61),
passing Order through, so the outputs recorded here -- column-major and
row-major -- are the reference's own.

The triangle of A that BLAS does not reference is filled with NaN (and so is
the diagonal for Diag = Unit, and the imaginary parts of a Hermitian diagonal
hold garbage): an implementation that reads them produces NaN or a wrong
value. Inputs are regenerated from their seeds by
``tests/golden_cases.symm_fill``; a checksum of the referenced entries guards
the generator.

Also recorded: the reference's xerbla_ lines for each illegal argument of
cblas_dsymm, cblas_zhemm, cblas_dtrmm, cblas_dtrsm (blas/dsymm.c:29-36,
blas/zhemm.c:30-41, blas/dtrmm.c:32-40, blas/dtrsm.c:31-38) and of their F77
wrappers (blas/dsymm.c:82-88, blas/zhemm.c:88-94, blas/dtrmm.c:76-84,
blas/dtrsm.c:86-94).

Run in a container that has the reference tree:  python tests/golden/make_golden_symm.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))
import oracle  # noqa: E402
from golden_cases import rank_k_fill, symm_fill  # noqa: E402
from make_golden import capture_stdout  # noqa: E402

OUT = os.path.join(HERE, "symm_trmm_golden.npz")
DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
SHAPES = [(1, 1), (7, 5), (33, 17), (20, 65)]
SIDE = {"L": 141, "R": 142}
UPLO = {"U": 121, "L": 122}
TRANS = {"N": 111, "T": 112, "C": 113}
DIAG = {"N": 131, "U": 132}


def scalars(tag, i):
    if tag in "sd":
        return [(1.5, -0.25), (-0.5, 0.0), (0.0, 2.0)][i % 3]
    return [(complex(1.5, -0.5), complex(-0.25, 0.75)), (complex(0.5, 1.0), 0j),
            (0j, complex(2.0, -1.0))][i % 3]


def checksum(A, B, C=None):
    parts = [np.nansum(A), np.nansum(B)] + ([np.nansum(C)] if C is not None else [])
    return np.array(parts, dtype=np.complex128)


def scalar_arg(tag, v):
    if tag == "s":
        return ctypes.c_float(v), None
    if tag == "d":
        return ctypes.c_double(v), None
    pair = np.array([complex(v).real, complex(v).imag], dtype=np.float32 if tag == "c" else np.float64)
    return pair.ctypes.data, pair


def main():
    ref = oracle.Reference()
    L = ref.L
    I, P = ctypes.c_int, ctypes.c_void_p
    for tag in "sdcz":
        sc = {"s": ctypes.c_float, "d": ctypes.c_double}.get(tag, P)
        kinds = ("symm", "hemm") if tag in "cz" else ("symm",)
        for kind in kinds:
            getattr(L, f"cblas_{tag}{kind}").argtypes = [I] * 5 + [sc, P, I, P, I, sc, P, I]
            getattr(L, f"{tag}{kind}_").argtypes = [P] * 12
        getattr(L, f"cblas_{tag}trmm").argtypes = [I] * 7 + [sc, P, I, P, I]
        getattr(L, f"{tag}trmm_").argtypes = [P] * 11
    rec = {}
    n = 0
    # SYMM / HEMM
    for tag in "sdcz":
        for kind in (("S", "symm"), ("H", "hemm")) if tag in "cz" else (("S", "symm"),):
            for (M, N) in SHAPES:
                for side in "LR":
                    for uplo in "UL":
                        for order in (102, 101):
                            if order == 101 and (M, N) != (7, 5):
                                continue
                            seed = 20000 + 10 * n
                            na = M if side == "L" else N
                            # row-major: ld >= max(M, N) also passes the reference's own check,
                            # which applies the column-major rule whatever the Order
                            rows_b = M if order == 102 else max(M, N)
                            lda, ldb, ldc = na + n % 2, rows_b + n % 3, rows_b + (n + 1) % 2
                            meta = [order, SIDE[side], UPLO[uplo], M, N, lda, ldb, ldc, seed]
                            x = symm_fill(kind[0], tag, meta)
                            C0 = x["C"].copy(order="F")
                            al, be = scalars(tag, n)
                            pa, ka = scalar_arg(tag, al)
                            pb, kb = scalar_arg(tag, be)
                            out = capture_stdout(lambda: getattr(L, f"cblas_{tag}{kind[1]}")(
                                order, SIDE[side], UPLO[uplo], M, N, pa, x["A"].ctypes.data, lda,
                                x["B"].ctypes.data, ldb, pb, x["C"].ctypes.data, ldc))
                            assert out == "", out
                            assert np.all(np.isfinite(x["C"])), (tag, kind, M, N, side, uplo, order)
                            key = f"{kind[1]}_{tag}_{n}"
                            rec[key + "_meta"] = np.array(meta, dtype=np.int64)
                            rec[key + "_scal"] = np.array([al, be], dtype=np.complex128)
                            rec[key + "_sum"] = checksum(x["A"], x["B"], C0)
                            rec[key + "_C"] = x["C"]
                            n += 1
    # TRMM
    for tag in "sdcz":
        for (M, N) in SHAPES[:3]:
            for side in "LR":
                for uplo in "UL":
                    for trans in ("NTC" if tag in "cz" else "NT"):
                        for diag in "NU":
                            for order in (102, 101):
                                if order == 101 and (M, N) != (7, 5):
                                    continue
                                seed = 20000 + 10 * n
                                na = M if side == "L" else N
                                rows_b = M if order == 102 else max(M, N)
                                lda, ldb = na + n % 3, rows_b + n % 2
                                meta = [order, SIDE[side], UPLO[uplo], TRANS[trans], DIAG[diag], M, N, lda, ldb,
                                        seed]
                                x = symm_fill("T", tag, meta)
                                B0 = x["B"].copy(order="F")
                                al = scalars(tag, n)[0] if n % 5 else (0.0 if tag in "sd" else 0j)
                                pa, ka = scalar_arg(tag, al)
                                out = capture_stdout(lambda: getattr(L, f"cblas_{tag}trmm")(
                                    order, SIDE[side], UPLO[uplo], TRANS[trans], DIAG[diag], M, N, pa,
                                    x["A"].ctypes.data, lda, x["B"].ctypes.data, ldb))
                                assert out == "", out
                                assert np.all(np.isfinite(x["B"])), (tag, M, N, side, uplo, trans, diag, order)
                                key = f"trmm_{tag}_{n}"
                                rec[key + "_meta"] = np.array(meta, dtype=np.int64)
                                rec[key + "_scal"] = np.array([al], dtype=np.complex128)
                                rec[key + "_sum"] = checksum(x["A"], B0)
                                rec[key + "_C"] = x["B"]
                                n += 1
    # TRSM (well-conditioned triangles, see golden_cases.symm_fill)
    for tag in "sdcz":
        getattr(L, f"cblas_{tag}trsm").argtypes = [I] * 7 + [{"s": ctypes.c_float, "d": ctypes.c_double}.get(tag, P),
                                                            P, I, P, I]
        for (M, N) in SHAPES[:3]:
            for side in "LR":
                for uplo in "UL":
                    for trans in ("NTC" if tag in "cz" else "NT"):
                        for diag in "NU":
                            for order in (102, 101):
                                if order == 101 and (M, N) != (7, 5):
                                    continue
                                seed = 20000 + 10 * n
                                na = M if side == "L" else N
                                rows_b = M if order == 102 else max(M, N)
                                lda, ldb = na + n % 3, rows_b + n % 2
                                meta = [order, SIDE[side], UPLO[uplo], TRANS[trans], DIAG[diag], M, N, lda, ldb,
                                        seed]
                                x = symm_fill("X", tag, meta)
                                B0 = x["B"].copy(order="F")
                                al = scalars(tag, n)[0] if n % 5 else (0.0 if tag in "sd" else 0j)
                                pa, ka = scalar_arg(tag, al)
                                out = capture_stdout(lambda: getattr(L, f"cblas_{tag}trsm")(
                                    order, SIDE[side], UPLO[uplo], TRANS[trans], DIAG[diag], M, N, pa,
                                    x["A"].ctypes.data, lda, x["B"].ctypes.data, ldb))
                                assert out == "", out
                                assert np.all(np.isfinite(x["B"])), (tag, M, N, side, uplo, trans, diag, order)
                                key = f"trsm_{tag}_{n}"
                                rec[key + "_meta"] = np.array(meta, dtype=np.int64)
                                rec[key + "_scal"] = np.array([al], dtype=np.complex128)
                                rec[key + "_sum"] = checksum(x["A"], B0)
                                rec[key + "_C"] = x["B"]
                                n += 1
    # HERK / HER2K (C/Z) and CSYRK / CSYR2K: C with NaN outside its triangle
    # and, for HERK, garbage imaginary parts on its diagonal (golden_cases.rank_k_fill)
    D_, F_ = ctypes.c_double, ctypes.c_float
    L.cblas_cherk.argtypes = [I] * 5 + [F_, P, I, F_, P, I]
    L.cblas_zherk.argtypes = [I] * 5 + [D_, P, I, D_, P, I]
    L.cblas_cher2k.argtypes = [I] * 5 + [P, P, I, P, I, F_, P, I]
    L.cblas_zher2k.argtypes = [I] * 5 + [P, P, I, P, I, D_, P, I]
    L.cblas_csyrk.argtypes = [I] * 5 + [P, P, I, P, P, I]
    L.cblas_csyr2k.argtypes = [I] * 5 + [P, P, I, P, I, P, P, I]
    for tag in "cz":
        for kind in ("herk", "her2k") + (("syrk", "syr2k") if tag == "c" else ()):
            herm = kind.startswith("her")
            for (N, K) in [(1, 1), (7, 3), (33, 65), (64, 17)]:
                for uplo in (121, 122):
                    for trans in (111, 113 if herm else 112):
                        for order in (102, 101):
                            if order == 101 and (N, K) != (7, 3):
                                continue
                            seed = 20000 + 10 * n
                            # the reference checks lda against the column-major rule whatever the Order
                            rows = N if trans == 111 else K
                            lda = (rows if order == 102 else max(N, K)) + n % 2
                            ldc = N + n % 3
                            meta = [order, uplo, trans, N, K, lda, lda + 1, ldc, seed]
                            x = rank_k_fill(kind, tag, meta)
                            C0 = x["C"].copy(order="F")
                            if kind == "herk":
                                al, be = [(1.5, -0.25), (0.0, 2.0), (-0.5, 0.0)][n % 3]
                                pa, pb = al, be
                            else:
                                al = [complex(1.5, -0.5), 0j, complex(0.5, 1.0)][n % 3]
                                be = -0.25 if herm else complex(-0.25, 0.75)
                                pa, ka = scalar_arg(tag, al)
                                pb, kb = (be, None) if herm else scalar_arg(tag, be)
                            fn = getattr(L, f"cblas_{tag}{kind}")
                            args = [order, uplo, trans, N, K, pa, x["A"].ctypes.data, lda]
                            if x["B"] is not None:
                                args += [x["B"].ctypes.data, lda + 1]
                            args += [pb, x["C"].ctypes.data, ldc]
                            out = capture_stdout(lambda: fn(*args))
                            assert out == "", out
                            key = f"{kind}_{tag}_{n}"
                            rec[key + "_meta"] = np.array(meta, dtype=np.int64)
                            rec[key + "_scal"] = np.array([al, be], dtype=np.complex128)
                            parts = [np.nansum(x["A"]), np.nansum(C0)] + (
                                [np.nansum(x["B"])] if x["B"] is not None else [])
                            rec[key + "_sum"] = np.array(parts, dtype=np.complex128)
                            rec[key + "_C"] = x["C"]
                            n += 1
    # xerbla lines
    A = np.zeros((4, 4)); B = np.zeros((4, 4)); C = np.ones((4, 4), order="F")
    Az = np.zeros((4, 4), dtype=np.complex128); Bz = Az.copy(); Cz = np.ones((4, 4), dtype=np.complex128, order="F")
    one = np.array([1.0, 0.0]); zero = np.array([0.0, 0.0])
    lines = []
    for info, kw in {1: dict(side=999), 2: dict(uplo=999), 3: dict(M=-1), 4: dict(N=-1), 7: dict(lda=2),
                     9: dict(ldb=2), 12: dict(ldc=2)}.items():
        a = dict(side=141, uplo=121, M=4, N=4, lda=4, ldb=4, ldc=4)
        a.update(kw)
        out = capture_stdout(lambda: L.cblas_dsymm(102, a["side"], a["uplo"], a["M"], a["N"], 1.0, A.ctypes.data,
                                                   a["lda"], B.ctypes.data, a["ldb"], 0.0, C.ctypes.data, a["ldc"]))
        lines.append(f"cblas_dsymm|{info}|{out}")
        out = capture_stdout(lambda: L.cblas_zhemm(102, a["side"], a["uplo"], a["M"], a["N"], one.ctypes.data,
                                                   Az.ctypes.data, a["lda"], Bz.ctypes.data, a["ldb"],
                                                   zero.ctypes.data, Cz.ctypes.data, a["ldc"]))
        lines.append(f"cblas_zhemm|{info}|{out}")
    for info, kw in {1: dict(side=999), 2: dict(uplo=999), 3: dict(trans=999), 4: dict(diag=999), 5: dict(M=-1),
                     6: dict(N=-1), 9: dict(lda=2), 11: dict(ldb=2)}.items():
        a = dict(side=141, uplo=121, trans=111, diag=131, M=4, N=4, lda=4, ldb=4)
        a.update(kw)
        out = capture_stdout(lambda: L.cblas_dtrmm(102, a["side"], a["uplo"], a["trans"], a["diag"], a["M"], a["N"],
                                                   1.0, A.ctypes.data, a["lda"], C.ctypes.data, a["ldb"]))
        lines.append(f"cblas_dtrmm|{info}|{out}")
        out = capture_stdout(lambda: L.cblas_dtrsm(102, a["side"], a["uplo"], a["trans"], a["diag"], a["M"], a["N"],
                                                   1.0, A.ctypes.data, a["lda"], C.ctypes.data, a["ldb"]))
        lines.append(f"cblas_dtrsm|{info}|{out}")
    r = ctypes.byref
    four = ctypes.c_int(4)
    al = ctypes.c_double(1.0); be = ctypes.c_double(0.0)
    for sd, up in [(b"X", b"U"), (b"L", b"Q"), (b"X", b"Q")]:
        cs, cu = ctypes.c_char(sd), ctypes.c_char(up)
        out = capture_stdout(lambda: L.dsymm_(r(cs), r(cu), r(four), r(four), r(al), A.ctypes.data, r(four),
                                              B.ctypes.data, r(four), r(be), C.ctypes.data, r(four)))
        lines.append(f"dsymm_{sd.decode()}{up.decode()}|-|{out}")
        out = capture_stdout(lambda: L.zhemm_(r(cs), r(cu), r(four), r(four), one.ctypes.data, Az.ctypes.data,
                                              r(four), Bz.ctypes.data, r(four), zero.ctypes.data, Cz.ctypes.data,
                                              r(four)))
        lines.append(f"zhemm_{sd.decode()}{up.decode()}|-|{out}")
    for chars in [(b"X", b"U", b"N", b"N"), (b"L", b"Q", b"N", b"N"), (b"L", b"U", b"Q", b"N"),
                  (b"L", b"U", b"N", b"Q"), (b"X", b"Q", b"Q", b"Q"), (b"L", b"U", b"Q", b"Q")]:
        cc = [ctypes.c_char(c) for c in chars]
        out = capture_stdout(lambda: L.dtrmm_(*(r(c) for c in cc), r(four), r(four), r(al), A.ctypes.data, r(four),
                                              C.ctypes.data, r(four)))
        lines.append(f"dtrmm_{b''.join(chars).decode()}|-|{out}")
        out = capture_stdout(lambda: L.dtrsm_(*(r(c) for c in cc), r(four), r(four), r(al), A.ctypes.data, r(four),
                                              C.ctypes.data, r(four)))
        lines.append(f"dtrsm_{b''.join(chars).decode()}|-|{out}")
    for info, kw in {1: dict(uplo=999), 2: dict(trans=112), 3: dict(N=-1), 4: dict(K=-1), 7: dict(lda=2),
                     10: dict(ldc=2)}.items():
        a = dict(uplo=121, trans=111, N=4, K=4, lda=4, ldc=4)
        a.update(kw)
        out = capture_stdout(lambda: L.cblas_zherk(102, a["uplo"], a["trans"], a["N"], a["K"], 1.0, Az.ctypes.data,
                                                   a["lda"], 0.0, Cz.ctypes.data, a["ldc"]))
        lines.append(f"cblas_zherk|{info}|{out}")
    for info, kw in {2: dict(trans=112), 9: dict(ldb=2), 12: dict(ldc=2)}.items():
        a = dict(trans=111, ldb=4, ldc=4)
        a.update(kw)
        out = capture_stdout(lambda: L.cblas_zher2k(102, 121, a["trans"], 4, 4, one.ctypes.data, Az.ctypes.data, 4,
                                                    Bz.ctypes.data, a["ldb"], 0.0, Cz.ctypes.data, a["ldc"]))
        lines.append(f"cblas_zher2k|{info}|{out}")
    L.zherk_.argtypes = [P] * 10
    for up, tr in [(b"X", b"N"), (b"U", b"Q"), (b"U", b"T")]:
        cu, ct = ctypes.c_char(up), ctypes.c_char(tr)
        alz, bez = ctypes.c_double(1.0), ctypes.c_double(0.0)
        out = capture_stdout(lambda: L.zherk_(r(cu), r(ct), r(four), r(four), r(alz), Az.ctypes.data, r(four),
                                              r(bez), Cz.ctypes.data, r(four)))
        lines.append(f"zherk_{up.decode()}{tr.decode()}|-|{out}")
    assert np.all(C == 1.0) and np.all(Cz == 1.0), "outputs must be untouched on argument errors"
    rec["xerbla"] = np.array(lines)
    np.savez_compressed(OUT, **rec)
    print(f"wrote {OUT}: {n} SYMM/HEMM/TRMM/TRSM/HERK/HER2K/CSYRK/CSYR2K cases + {len(lines)} xerbla lines")


if __name__ == "__main__":
    main()
