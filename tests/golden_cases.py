"""Helpers that rebuild the golden cases (inputs from their seeds)."""
import re

import numpy as np

import oracle

DT = {"d": np.float64, "s": np.float32, "z": np.complex128, "c": np.complex64}


GEMM_KEY = re.compile(r"^([dszc])_(\d+)_meta$")  # "<tag>_<n>_meta"; SYRK cases use their own prefixes


def cases(golden, tags=("d", "s", "z")):
    keys = sorted({k.rsplit("_", 1)[0] for k in golden.files
                   if GEMM_KEY.match(k) and GEMM_KEY.match(k).group(1) in tags},
                  key=lambda s: (s[0], int(s.split("_")[1])))
    for key in keys:
        if key.startswith("edge"):
            continue
        tag = key.split("_")[0]
        dt = DT[tag]
        M, N, K, lda, ldb, ldc, ta, tb = (int(v) for v in golden[key + "_meta"])
        ta, tb = chr(ta), chr(tb)
        al, be = golden[key + "_scal"]
        if dt not in (np.complex128, np.complex64):
            al, be = float(al.real), float(be.real)
        else:
            al, be = complex(al), complex(be)
        seed = int(golden[key + "_seed"][0])
        ra, ca = oracle.shape_of_op(ta, M, K)
        rb, cb = oracle.shape_of_op(tb, K, N)
        A = oracle.uniform((lda, ca), dt, seed)
        B = oracle.uniform((ldb, cb), dt, seed + 1)
        C0 = oracle.uniform((ldc, N), dt, seed + 2)
        yield dict(key=key, dt=dt, M=M, N=N, K=K, lda=lda, ldb=ldb, ldc=ldc, ta=ta, tb=tb, alpha=al,
                   beta=be, A=A, B=B, C0=C0, C=golden[key + "_C"], sums=golden[key + "_sum"])


def edge_cases(golden):
    for case in range(3):
        key = f"edge_{case}"
        M, N, K, lda, ldb, ldc, ta, tb = (int(v) for v in golden[key + "_meta"])
        al, be = golden[key + "_scal"]
        yield dict(key=key, M=M, N=N, K=K, lda=lda, ldb=ldb, ldc=ldc, alpha=float(al.real),
                   beta=float(be.real), A=golden[key + "_A"], B=golden[key + "_B"],
                   C0=golden[key + "_C0"], C=golden[key + "_C"])


def tol_ratio(case, got):
    """max |got - C_ref| / ((K+2) u (|alpha||A||B| + |beta||C0|)) over the case's C.

    (K+2) u: K roundings in the dot product, one for alpha, one for the beta term;
    complex doubles it (four real products per complex multiply-add)."""
    dt = case["dt"]
    M, N, K = case["M"], case["N"], case["K"]
    ta, tb = case["ta"], case["tb"]
    ra, ca = oracle.shape_of_op(ta, M, K)
    rb, cb = oracle.shape_of_op(tb, K, N)
    Av, Bv = case["A"][:ra, :ca], case["B"][:rb, :cb]
    opA = Av if ta == "N" else (Av.T if ta == "T" else np.conj(Av.T))
    opB = Bv if tb == "N" else (Bv.T if tb == "T" else np.conj(Bv.T))
    bound = abs(case["alpha"]) * (np.abs(opA).astype(np.float64) @ np.abs(opB).astype(np.float64))
    if case["beta"] != 0:
        bound = bound + abs(case["beta"]) * np.abs(case["C0"][:M, :N]).astype(np.float64)
    u = oracle.UNIT_ROUNDOFF[np.dtype(dt).type]
    gamma = (K + 2) * u * (2.0 if dt in (np.complex128, np.complex64) else 1.0)
    err = np.abs(got[:M, :N].astype(np.complex128) - case["C"][:M, :N].astype(np.complex128))
    scale = np.maximum(bound, np.finfo(np.float64).tiny)
    return float(np.max(err / (gamma * scale))) if err.size else 0.0


# ---- SYMM / HEMM / TRMM fixtures (tests/golden/symm_trmm_golden.npz) --------

SYMM_GOLDEN_DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
SIDE_OF = {141: "L", 142: "R"}
UPLO_OF = {121: "U", 122: "L"}
TRANS_OF = {111: "N", 112: "T", 113: "C"}
DIAG_OF = {131: "N", 132: "U"}


def poison(kind, uplo, A, na, diag="N"):
    """NaN in the entries of A that BLAS does not reference: the triangle
    opposite uplo, the diagonal for Diag = Unit; the imaginary parts of a
    Hermitian diagonal get a nonzero value that BLAS must ignore."""
    i, j = np.indices((na, na))
    hidden = (i > j) if uplo == "U" else (i < j)
    V = A[:na, :na]
    V[hidden] = np.nan
    if kind == "T" and diag == "U":
        np.fill_diagonal(V, np.nan)
    if kind == "H":
        d = np.diag(V).copy()
        np.fill_diagonal(V, d.real + 1j * 0.375)


def symm_fill(kind, tag, meta):
    """Inputs of one SYMM / HEMM (kind 'S' / 'H'), TRMM ('T') or TRSM ('X')
    case from its meta row, and the column-major form of the problem.
      'S' / 'H': meta = order, side, uplo, M, N, lda, ldb, ldc, seed
      'T' / 'X': meta = order, side, uplo, trans, diag, M, N, lda, ldb, seed
    TRSM's triangle is made well conditioned: off-diagonal entries
    U[-1, 1] / order, diagonal 2 + U[-1, 1] / order.
    Arrays are Fortran-ordered with the leading dimension first: a row-major
    (101) matrix with r rows and leading dimension ld is the array of shape
    (ld, r), whose columns are the matrix's rows. The column-major problem of
    a row-major call has side and uplo flipped and M, N swapped."""
    dt = SYMM_GOLDEN_DT[tag]
    meta = [int(v) for v in meta]
    if kind in "SH":
        order, side, uplo, M, N, lda, ldb, ldc, seed = meta
        trans, diag = 111, 131
    else:
        order, side, uplo, trans, diag, M, N, lda, ldb, seed = meta
        ldc = ldb
    rm = order == 101
    side_s, uplo_s = SIDE_OF[side], UPLO_OF[uplo]
    cm = dict(side=side_s, uplo=uplo_s, M=M, N=N, trans=TRANS_OF[trans], diag=DIAG_OF[diag])
    if rm:
        cm.update(side="R" if side_s == "L" else "L", uplo="L" if uplo_s == "U" else "U", M=N, N=M)
    na = cm["M"] if cm["side"] == "L" else cm["N"]
    A = oracle.uniform((lda, na), dt, seed)
    if kind == "X":
        A /= na
        A[np.arange(na), np.arange(na)] += 2
    poison("T" if kind == "X" else kind, cm["uplo"], A, na, cm["diag"])
    B = oracle.uniform((ldb, cm["N"]), dt, seed + 1)
    out = dict(order=order, side=side, uplo=uplo, trans=trans, diag=diag, M=M, N=N, lda=lda, ldb=ldb,
               ldc=ldc, A=A, B=B, na=na, cm=cm, dt=dt)
    if kind in "SH":
        out["C"] = oracle.uniform((ldc, cm["N"]), dt, seed + 2)
    return out


def symm_checksum(x):
    parts = [np.nansum(x["A"]), np.nansum(x["B"])] + ([np.nansum(x["C"])] if "C" in x else [])
    return np.array(parts, dtype=np.complex128)


def symm_keys(golden, prefix):
    return sorted({k.rsplit("_", 1)[0] for k in golden.files if k.startswith(prefix)},
                  key=lambda k: int(k.split("_")[-1]))


def symm_case(golden, key):
    """(kind, tag, inputs, alpha, beta, reference output) of one fixture key."""
    kind = {"symm": "S", "hemm": "H", "trmm": "T", "trsm": "X"}[key.split("_")[0]]
    tag = key.split("_")[1]
    x = symm_fill(kind, tag, golden[key + "_meta"])
    assert np.allclose(symm_checksum(x), golden[key + "_sum"]), "fixture generator changed"
    sc = golden[key + "_scal"]
    real = tag in "sd"
    al = float(sc[0].real) if real else complex(sc[0])
    be = (float(sc[1].real) if real else complex(sc[1])) if kind in "SH" else None
    return kind, tag, x, al, be, golden[key + "_C"]


def trsm_bound(x, al, X):
    """Componentwise forward-error bound of a triangular solve against the
    solution X (both sides' roundings): 2 (K + 2) u |T^-1| (|T| |X| + |alpha B|)
    (left, T = op(A)), mirrored for the right side; twice that for complex."""
    cm, na = x["cm"], x["na"]
    M, N = cm["M"], cm["N"]
    dt = x["dt"]
    cplx = np.issubdtype(dt, np.complexfloating)
    wide = np.complex128 if cplx else np.float64
    T = oracle.complete("T", cm["uplo"], x["A"], na, cm["diag"]).astype(wide)
    T = {"N": T, "T": T.T, "C": T.conj().T}[cm["trans"]]
    aTi = np.abs(np.linalg.inv(T))
    aT, aX = np.abs(T), np.abs(X[:M, :N].astype(wide))
    aB = abs(al) * np.abs(x["B"][:M, :N].astype(wide))
    scale = aTi @ (aT @ aX + aB) if cm["side"] == "L" else (aX @ aT + aB) @ aTi
    u = oracle.UNIT_ROUNDOFF[np.dtype(dt).type]
    return 2 * (na + 2) * u * (2.0 if cplx else 1.0) * scale


def symm_bound(kind, x, al, be):
    """Componentwise bound on |computed - reference| over the column-major
    output block: both results carry at most (K + 2) u (|alpha| |op(A)| |B| +
    |beta| |C0|) each (twice that for complex), K the order of A."""
    cm, na = x["cm"], x["na"]
    M, N = cm["M"], cm["N"]
    Af = oracle.complete({"S": "S", "H": "H", "T": "T"}[kind], cm["uplo"], x["A"], na, cm["diag"])
    aA = np.abs(Af).astype(np.float64)
    if cm["trans"] != "N":
        aA = aA.T
    aB = np.abs(x["B"][:M, :N]).astype(np.float64)
    prod = aA @ aB if cm["side"] == "L" else aB @ aA
    bound = abs(al) * prod
    if kind in "SH" and be != 0:
        bound = bound + abs(be) * np.abs(x["C"][:M, :N]).astype(np.float64)
    dt = x["dt"]
    u = oracle.UNIT_ROUNDOFF[np.dtype(dt).type]
    cplx = np.issubdtype(dt, np.complexfloating)
    return 2 * (na + 2) * u * (2.0 if cplx else 1.0) * bound


def symm_oracle(kind, x, al, be):
    """The oracle's result for one case, on copies (column-major problem)."""
    cm = x["cm"]
    if kind in "SH":
        C = x["C"].copy(order="F")
        return oracle.symm(cm["side"], cm["uplo"], cm["M"], cm["N"], al, x["A"], x["lda"], x["B"], x["ldb"], be,
                           C, x["ldc"], herm=kind == "H")
    B = x["B"].copy(order="F")
    if kind == "X":
        return oracle.trsm(cm["side"], cm["uplo"], cm["trans"], cm["diag"], cm["M"], cm["N"], al, x["A"], x["lda"],
                           B, x["ldb"])
    return oracle.trmm(cm["side"], cm["uplo"], cm["trans"], cm["diag"], cm["M"], cm["N"], al, x["A"], x["lda"], B,
                       x["ldb"])


def symm_check(kind, x, got, want, al, be):
    """got against the reference output: the M x N block (column-major view)
    within the bound, finite, and every padding row exactly the input."""
    cm = x["cm"]
    M, N = cm["M"], cm["N"]
    before = x["C"] if kind in "SH" else x["B"]
    assert np.array_equal(got[M:], before[M:], equal_nan=True)
    blk = got[:M, :N]
    assert np.all(np.isfinite(blk)), "a non-referenced entry of A was read"
    err = np.abs(blk.astype(np.complex128) - want[:M, :N].astype(np.complex128))
    bound = trsm_bound(x, al, want) if kind == "X" else symm_bound(kind, x, al, be)
    assert np.all(err <= bound), float(np.max(err / np.maximum(bound, 1e-300)))


# ---- HERK / HER2K (C/Z) and CSYRK / CSYR2K fixtures ---------------------------
# meta = order, uplo, trans, N, K, lda, ldb, ldc, seed. The column-major problem
# of a row-major call has uplo flipped and NoTrans / (Conj)Trans swapped.

def rank_k_fill(kind, tag, meta):
    """Inputs of one 'herk', 'her2k', 'syrk' or 'syr2k' case: A (and B), C
    with NaN in the triangle BLAS does not reference and, for the Hermitian
    kinds, a nonzero imaginary part on C's diagonal (which BLAS takes as
    zero)."""
    dt = SYMM_GOLDEN_DT[tag]
    order, uplo, trans, N, K, lda, ldb, ldc, seed = (int(v) for v in meta)
    herm = kind.startswith("her")
    rm = order == 101
    cm_uplo = UPLO_OF[uplo] if not rm else ("L" if uplo == 121 else "U")
    ctr = "C" if herm else "T"
    cm_trans = ("N" if trans == 111 else ctr) if not rm else (ctr if trans == 111 else "N")
    cols = K if cm_trans == "N" else N
    A = oracle.uniform((lda, cols), dt, seed)
    B = oracle.uniform((ldb, cols), dt, seed + 1) if kind.endswith("2k") else None
    C = oracle.uniform((ldc, N), dt, seed + 2)
    i, j = np.indices((N, N))
    C[:N, :N][(i > j) if cm_uplo == "U" else (i < j)] = np.nan
    if herm:
        d = np.arange(N)
        C[d, d] = C[d, d].real + 0.375j
    return dict(A=A, B=B, C=C, N=N, K=K, lda=lda, ldb=ldb, ldc=ldc, uplo=uplo, trans=trans, order=order,
                cm_uplo=cm_uplo, cm_trans=cm_trans, dt=dt, kind=kind)


def rank_k_case(golden, key):
    kind, tag = key.split("_")[0], key.split("_")[1]
    x = rank_k_fill(kind, tag, golden[key + "_meta"])
    parts = [np.nansum(x["A"]), np.nansum(x["C"])] + ([np.nansum(x["B"])] if x["B"] is not None else [])
    assert np.allclose(np.array(parts, dtype=np.complex128), golden[key + "_sum"]), "fixture generator changed"
    al, be = (complex(v) for v in golden[key + "_scal"])
    if kind == "herk":
        al, be = al.real, be.real
    elif kind == "her2k":
        be = be.real
    return kind, tag, x, al, be, golden[key + "_C"]


def rank_k_oracle(x, al, be):
    C = x["C"].copy(order="F")
    B, ldb = (x["B"], x["ldb"]) if x["B"] is not None else (None, None)
    if x["kind"].startswith("her"):
        if x["kind"] == "her2k" and x["order"] == 101:  # the transposed problem's alpha is conj(alpha)
            al = np.conj(al)
        return oracle.herk(x["cm_uplo"], x["cm_trans"], x["N"], x["K"], al, x["A"], x["lda"], be, C, x["ldc"], B, ldb)
    return oracle.syrk(x["cm_uplo"], x["cm_trans"], x["N"], x["K"], al, x["A"], x["lda"], be, C, x["ldc"], B, ldb)


def rank_k_check(x, got, want, al, be):
    """The uplo triangle within the componentwise bound, the other triangle and
    the rows beyond N unchanged (NaN included), a real diagonal for HERK."""
    N, K = x["N"], x["K"]
    C0 = x["C"]
    m = oracle.tri_mask(x["cm_uplo"], N)
    assert np.array_equal(got[N:], C0[N:], equal_nan=True)
    assert np.array_equal(got[:N, :N][~m], C0[:N, :N][~m], equal_nan=True)
    if x["kind"].startswith("her"):
        assert np.all(np.diag(got[:N, :N]).imag == 0)
    wide = np.complex128
    A = x["A"].astype(wide)
    opA = A[:N, :K] if x["cm_trans"] == "N" else (A[:K, :N].conj().T if x["cm_trans"] == "C" else A[:K, :N].T)
    if x["B"] is not None:
        Bw = x["B"].astype(wide)
        opB = Bw[:N, :K] if x["cm_trans"] == "N" else Bw[:K, :N].T
        prod = np.abs(opA) @ np.abs(opB).T + np.abs(opB) @ np.abs(opA).T
    else:
        prod = np.abs(opA) @ np.abs(opA).T
    c0 = np.nan_to_num(np.abs(C0[:N, :N].astype(wide)))
    u = oracle.UNIT_ROUNDOFF[np.dtype(x["dt"]).type]
    bound = 2 * 2 * (K + 2) * u * (abs(al) * prod + abs(be) * c0)
    err = np.abs(got[:N, :N].astype(wide) - want[:N, :N].astype(wide))[m]
    assert np.all(err <= bound[m]), float(np.max(err / np.maximum(bound[m], 1e-300)))
