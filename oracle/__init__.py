"""CPU oracle for the GEMM path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs import this package, and only to check results: nothing in
``blasx_b200`` imports it, and the shipped library never routes through it.

It wraps ``oracle/liboracle.so`` (built by ``oracle/Makefile``):

* ``gemm_tiled``  -- plain-C restatement of the reference's tiled GEMM
  (blas/blasx_dgemm.c:5-96 and :251-356, margin_adjustment in
  blas/blasx_mem_control.c:24-42);
* ``dd_entries``  -- double-double (Ogita-Rump-Oishi Dot2) value of sampled C
  entries plus the componentwise bound scale |alpha||A||B| + |beta||C0|;
* ``OpenBLAS``    -- the CPU BLAS the reference dispatches to
  (blas/blasx_internal.c:26-36), found with dlopen over a candidate list;
* ``Reference``   -- the reference library itself, compiled from its own
  sources into ``oracle/_ref`` (CPU path only for dims <= 1000,
  blas/dgemm.c:61-64).

Parity of this oracle is pinned against ``tests/golden`` (outputs of the
reference library run on its CPU path, generated by
``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess
import sysconfig

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libblasx_ref.so")

NOTRANS, TRANS, CONJTRANS = 111, 112, 113
ROWMAJOR, COLMAJOR = 101, 102
TRANS_OF = {"N": NOTRANS, "T": TRANS, "C": CONJTRANS}

# machine epsilons (unit roundoff) per dtype
UNIT_ROUNDOFF = {np.float64: 2.0 ** -53, np.float32: 2.0 ** -24, np.complex128: 2.0 ** -53,
                 np.complex64: 2.0 ** -24}

_lib = None
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_F = ctypes.c_float


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_dgemm_tiled.argtypes = [_I] * 5 + [_D, _P, _I, _P, _I, _D, _P, _I, _I]
        L.oracle_sgemm_tiled.argtypes = [_I] * 5 + [_F, _P, _I, _P, _I, _F, _P, _I, _I]
        L.oracle_zgemm_tiled.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _P, _P, _I, _I]
        L.oracle_cgemm_tiled.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _P, _P, _I, _I]
        L.oracle_dgemm_dd_entries.argtypes = [_I] * 5 + [_D, _P, _I, _P, _I, _D, _P, _I, _I64, _P, _P, _P, _P, _P]
        L.oracle_sgemm_dd_entries.argtypes = [_I] * 5 + [_F, _P, _I, _P, _I, _F, _P, _I, _I64, _P, _P, _P, _P, _P]
        L.oracle_zgemm_dd_entries.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _P, _P, _I, _I64, _P, _P, _P, _P, _P]
        L.oracle_openblas_open.argtypes = [ctypes.c_char_p]
        L.oracle_openblas_name.restype = ctypes.c_char_p
        L.oracle_openblas_dgemm.argtypes = [_I] * 6 + [_D, _P, _I, _P, _I, _D, _P, _I]
        L.oracle_openblas_sgemm.argtypes = [_I] * 6 + [_F, _P, _I, _P, _I, _F, _P, _I]
        L.oracle_openblas_zgemm.argtypes = [_I] * 6 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.oracle_openblas_cgemm.argtypes = [_I] * 6 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.oracle_fill_uniform_f64.argtypes = [_P, _I64, ctypes.c_uint64, _D, _D]
        L.oracle_fill_uniform_f32.argtypes = [_P, _I64, ctypes.c_uint64, _F, _F]
        L.oracle_fill_spread_f64.argtypes = [_P, _I64, ctypes.c_uint64, _D]
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def shape_of_op(trans: str, rows: int, cols: int) -> tuple[int, int]:
    """Stored (column-major) shape of an operand whose op() is rows x cols."""
    return (rows, cols) if trans == "N" else (cols, rows)


# --------------------------------------------------------------------------
# generators (column-major, Fortran-ordered numpy arrays)
# --------------------------------------------------------------------------

def uniform(shape, dtype, seed: int, lo=-1.0, hi=1.0) -> np.ndarray:
    """Seeded U[lo,hi] column-major matrix (SplitMix64 counter RNG)."""
    dtype = np.dtype(dtype)
    if dtype in (np.complex128, np.complex64):
        part = np.float64 if dtype == np.complex128 else np.float32
        re = uniform(shape, part, seed, lo, hi)
        im = uniform(shape, part, seed ^ 0x9E3779B9, lo, hi)
        out = np.empty(shape, dtype=dtype, order="F")
        out.real, out.imag = re, im
        return out
    out = np.empty(shape, dtype=dtype, order="F")
    n = out.size
    if dtype == np.float64:
        lib().oracle_fill_uniform_f64(_ptr(out), n, seed, lo, hi)
    elif dtype == np.float32:
        lib().oracle_fill_uniform_f32(_ptr(out), n, seed, lo, hi)
    else:
        raise TypeError(dtype)
    return out


def spread(shape, seed: int, phi: float) -> np.ndarray:
    """Seeded U[-0.5,0.5]*exp(phi*g), g~N(0,1), float64 column-major."""
    out = np.empty(shape, dtype=np.float64, order="F")
    lib().oracle_fill_spread_f64(_ptr(out), out.size, seed, phi)
    return out


# --------------------------------------------------------------------------
# tiled restatement and double-double entries
# --------------------------------------------------------------------------

def gemm_tiled(transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, block_dim=2048):
    """Reference-algorithm GEMM on CPU; updates C (Fortran array) in place."""
    ta, tb = TRANS_OF[transa], TRANS_OF[transb]
    L = lib()
    if C.dtype == np.float64:
        L.oracle_dgemm_tiled(ta, tb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C), ldc, block_dim)
    elif C.dtype == np.float32:
        L.oracle_sgemm_tiled(ta, tb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C), ldc, block_dim)
    elif C.dtype == np.complex64:
        al = np.array([complex(alpha).real, complex(alpha).imag], dtype=np.float32)
        be = np.array([complex(beta).real, complex(beta).imag], dtype=np.float32)
        L.oracle_cgemm_tiled(ta, tb, M, N, K, _ptr(al), _ptr(A), lda, _ptr(B), ldb, _ptr(be), _ptr(C), ldc,
                             block_dim)
    elif C.dtype == np.complex128:
        al = np.array([complex(alpha).real, complex(alpha).imag])
        be = np.array([complex(beta).real, complex(beta).imag])
        L.oracle_zgemm_tiled(ta, tb, M, N, K, _ptr(al), _ptr(A), lda, _ptr(B), ldb, _ptr(be), _ptr(C), ldc, block_dim)
    else:
        raise TypeError(C.dtype)
    return C


def tri_mask(uplo: str, N: int) -> np.ndarray:
    """Boolean N x N mask of the entries ?SYRK / ?SYR2K update ('U': i <= j)."""
    i, j = np.indices((N, N))
    return i <= j if uplo == "U" else i >= j


def syrk(uplo, trans, N, K, alpha, A, lda, beta, C, ldc, B=None, ldb=None):
    """Restatement of BLAS ?SYRK (B None) and ?SYR2K, the operations the
    reference hands to its CPU BLAS (blas/dsyrk.c:60-66, blas/dsyr2k.c:61-70):
    C <- alpha op(A) op(A)^T + beta C, or alpha op(A) op(B)^T + alpha op(B)
    op(A)^T + beta C, on the uplo triangle only; op(X) = X (trans 'N') or X^T.
    Computed as tiled GEMMs on a copy of C whose triangle is copied back."""
    ta, tb = ("N", "T") if trans == "N" else ("T", "N")
    full = C.copy(order="F")
    if B is None:
        gemm_tiled(ta, tb, N, N, K, alpha, A, lda, A, lda, beta, full, ldc)
    else:
        gemm_tiled(ta, tb, N, N, K, alpha, A, lda, B, ldb, beta, full, ldc)
        gemm_tiled(ta, tb, N, N, K, alpha, B, ldb, A, lda, 1.0, full, ldc)
    m = tri_mask(uplo, N)
    view, fv = C[:N, :N], full[:N, :N]
    view[m] = fv[m]
    return C


def herk(uplo, trans, N, K, alpha, A, lda, beta, C, ldc, B=None, ldb=None):
    """Restatement of BLAS ?HERK (B None) and ?HER2K, which the reference
    hands to its CPU BLAS (blas/zherk.c:44-77, blas/zher2k.c:50-86): C <-
    alpha op(A) op(A)^H + beta C, or alpha op(A) op(B)^H + conj(alpha) op(B)
    op(A)^H + beta C, on the uplo triangle only, op(X) = X (trans 'N') or
    X^H ('C'); the imaginary parts of C's diagonal are taken as zero on input
    and set to zero on output. Tiled GEMMs on a copy of C whose triangle is
    copied back."""
    ta, tb = ("N", "C") if trans == "N" else ("C", "N")
    full = C.copy(order="F")
    if B is None:
        gemm_tiled(ta, tb, N, N, K, alpha, A, lda, A, lda, beta, full, ldc)
    else:
        gemm_tiled(ta, tb, N, N, K, alpha, A, lda, B, ldb, beta, full, ldc)
        gemm_tiled(ta, tb, N, N, K, np.conj(alpha), B, ldb, A, lda, 1.0, full, ldc)
    m = tri_mask(uplo, N)
    view, fv = C[:N, :N], full[:N, :N]
    view[m] = fv[m]
    d = np.arange(N)
    view[d, d] = view[d, d].real
    return C


def complete(kind, uplo, X, n, diag="N"):
    """The full n x n matrix that BLAS reads from the uplo triangle of X:
    kind 'S' symmetric (mirror), 'H' Hermitian (conjugate mirror, the
    imaginary parts of the diagonal taken as zero), 'T' triangular (zero
    outside, ones on the diagonal when diag is 'U'). Entries outside the
    triangle of X are never read. Returns a new Fortran-ordered array."""
    S = np.array(X[:n, :n], order="F")
    keep = tri_mask(uplo, n)
    strict = keep & ~np.eye(n, dtype=bool)
    if kind == "T":
        S[~keep] = 0
        if diag == "U":
            np.fill_diagonal(S, 1)
        return S
    other = S.T.conj() if kind == "H" else S.T
    S = np.where(strict, S, np.where(strict.T, other, S))
    if kind == "H":
        np.fill_diagonal(S, np.diag(S).real)
    return np.asfortranarray(S)


def symm(side, uplo, M, N, alpha, A, lda, B, ldb, beta, C, ldc, herm=False):
    """Restatement of BLAS ?SYMM / ?HEMM, which the reference hands to its CPU
    BLAS for every size (blas/dsymm.c:44-57, blas/zhemm.c): C <- alpha A B +
    beta C (side 'L', A M x M) or alpha B A + beta C (side 'R', A N x N), A
    read from its uplo triangle only. A tiled GEMM on the completed A."""
    na = M if side == "L" else N
    Af = complete("H" if herm else "S", uplo, A, na)
    if side == "L":
        gemm_tiled("N", "N", M, N, M, alpha, Af, na, B, ldb, beta, C, ldc)
    else:
        gemm_tiled("N", "N", M, N, N, alpha, B, ldb, Af, na, beta, C, ldc)
    return C


def trmm(side, uplo, transa, diag, M, N, alpha, A, lda, B, ldb):
    """Restatement of BLAS ?TRMM, which the reference hands to its CPU BLAS
    (blas/dtrmm.c:43-60): B <- alpha op(A) B (side 'L', A M x M) or alpha B
    op(A) ('R', A N x N), A triangular (uplo, diag), op(A) = A, A^T or A^H.
    A tiled GEMM on the completed A into a fresh buffer, copied into B."""
    na = M if side == "L" else N
    Af = complete("T", uplo, A, na, diag)
    Bin = np.array(B[:M, :N], order="F")
    out = np.zeros((M, N), dtype=B.dtype, order="F")
    if side == "L":
        gemm_tiled(transa, "N", M, N, M, alpha, Af, na, Bin, M, 0.0, out, M)
    else:
        gemm_tiled("N", transa, M, N, N, alpha, Bin, M, Af, na, 0.0, out, M)
    B[:M, :N] = out
    return B


def trsm(side, uplo, transa, diag, M, N, alpha, A, lda, B, ldb):
    """Restatement of BLAS ?TRSM, which the reference hands to its CPU BLAS
    (blas/dtrsm.c:44-61): solves op(A) X = alpha B (side 'L', A M x M) or
    X op(A) = alpha B ('R', A N x N) for X, which overwrites B; A triangular
    (uplo, diag), only its uplo triangle read. Column-oriented substitution
    as in reference BLAS, vectorised over the right-hand sides; in float64 /
    complex128 whatever the input type, rounded to B's type at the end."""
    na = M if side == "L" else N
    wide = np.complex128 if np.iscomplexobj(B) else np.float64
    T = complete("T", uplo, A, na, diag).astype(wide)
    if transa == "T":
        T = T.T
    elif transa == "C":
        T = T.conj().T
    X = alpha * np.array(B[:M, :N], dtype=wide)
    if side == "R":  # X op(A) = alpha B  <=>  op(A)^T X^T = alpha B^T
        T, X = T.T, X.T
    n = T.shape[0]
    # the system matrix is op(A) (left) or op(A)^T (right): lower when the
    # stored triangle, transposed or not, ends up below the diagonal
    lower = (uplo == "L") == ((transa == "N") == (side == "L"))
    order = range(n) if lower else range(n - 1, -1, -1)
    for k in order:
        if diag != "U":
            X[k, :] /= T[k, k]
        rest = slice(k + 1, n) if lower else slice(0, k)
        X[rest, :] -= np.outer(T[rest, k], X[k, :])
    if side == "R":
        X = X.T
    B[:M, :N] = X.astype(B.dtype)
    return B


def dd_entries(transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C0, ldc, ii, jj):
    """Double-double values of sampled entries of alpha*op(A)op(B)+beta*C0.

    Returns (value, bound): value as float64 (or complex128) rounded from the
    double-double, bound = |alpha| sum_k |a_ik||b_kj| + |beta||c0_ij|.
    """
    ta, tb = TRANS_OF[transa], TRANS_OF[transb]
    ii = np.ascontiguousarray(ii, dtype=np.int64)
    jj = np.ascontiguousarray(jj, dtype=np.int64)
    n = ii.size
    L = lib()
    if A.dtype == np.complex64:  # products of floats are exact in double: widen and use the complex128 sums
        A = np.asfortranarray(A, dtype=np.complex128)
        B = np.asfortranarray(B, dtype=np.complex128)
        C0 = None if C0 is None else np.asfortranarray(C0, dtype=np.complex128)
    c0p = _ptr(C0) if (C0 is not None and beta != 0) else None
    if A.dtype == np.complex128:
        hi = np.empty(2 * n); lo = np.empty(2 * n); bd = np.empty(2 * n)
        al = np.array([complex(alpha).real, complex(alpha).imag])
        be = np.array([complex(beta).real, complex(beta).imag])
        L.oracle_zgemm_dd_entries(ta, tb, M, N, K, _ptr(al), _ptr(A), lda, _ptr(B), ldb, _ptr(be),
                                  c0p, ldc, n, _ptr(ii), _ptr(jj), _ptr(hi), _ptr(lo), _ptr(bd))
        v = (hi + lo)
        return v[0::2] + 1j * v[1::2], bd[0::2]
    hi = np.empty(n); lo = np.empty(n); bd = np.empty(n)
    if A.dtype == np.float64:
        L.oracle_dgemm_dd_entries(ta, tb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta,
                                  c0p, ldc, n, _ptr(ii), _ptr(jj), _ptr(hi), _ptr(lo), _ptr(bd))
    elif A.dtype == np.float32:
        L.oracle_sgemm_dd_entries(ta, tb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta,
                                  c0p, ldc, n, _ptr(ii), _ptr(jj), _ptr(hi), _ptr(lo), _ptr(bd))
    else:
        raise TypeError(A.dtype)
    return hi + lo, bd


def componentwise_ratio(C, ii, jj, ref, bound, K, dtype):
    """max_ij |C_ij - C*_ij| / (gamma * bound_ij), gamma = (K+2)*u (u of dtype).

    A ratio <= 1 means every sampled entry meets the componentwise bound
    |C - C*| <= (K+2) u (|alpha||A||B| + |beta||C0|): K roundings in the dot
    product, one for alpha and one for the beta term; complex doubles gamma.
    Returns (ratio, max_normalised_error) where the latter is
    max |C - C*| / bound (the "measured error" reported per run).
    """
    u = UNIT_ROUNDOFF[np.dtype(dtype).type]
    got = np.asarray(C)[ii, jj].astype(np.complex128 if np.iscomplexobj(C) else np.float64)
    err = np.abs(got - ref)
    gamma = (K + 2) * u * (2.0 if np.iscomplexobj(C) else 1.0)
    scale = np.where(bound > 0, bound, np.finfo(np.float64).tiny)
    norm = err / scale
    return float(np.max(norm / gamma)) if norm.size else 0.0, float(np.max(norm)) if norm.size else 0.0


# --------------------------------------------------------------------------
# OpenBLAS (the reference's CPU BLAS) and the reference library itself
# --------------------------------------------------------------------------

def _site() -> str:
    return sysconfig.get_paths()["purelib"]


def openblas_candidates() -> str:
    """':'-separated 'path|prefix|ilp64' list, newest OpenBLAS first."""
    site = _site()
    cands = []
    env = os.environ.get("BLASX_ORACLE_OPENBLAS")
    if env:
        cands.append(env)
    for p in sorted(glob.glob(os.path.join(site, "numpy.libs", "libscipy_openblas64_*.so"))):
        cands.append(f"{p}|scipy_|1")
    for p in sorted(glob.glob(os.path.join(site, "scipy.libs", "libscipy_openblas-*.so"))):
        cands.append(f"{p}|scipy_|0")
    for p in sorted(glob.glob(os.path.join(site, "opencv_python_headless.libs", "libopenblasp-*.so"))):
        cands.append(f"{p}||0")
    return ":".join(cands)


def _preload_gfortran(directory: str) -> None:
    for pat in ("libquadmath*", "libgfortran*"):
        for f in sorted(glob.glob(os.path.join(directory, pat))):
            try:
                ctypes.CDLL(f, mode=ctypes.RTLD_GLOBAL)
            except OSError:
                pass


class OpenBLAS:
    """OpenBLAS cblas_?gemm through the oracle's dlopen wrapper."""

    def __init__(self):
        for d in ("numpy.libs", "scipy.libs", "opencv_python_headless.libs"):
            _preload_gfortran(os.path.join(_site(), d))
        L = lib()
        if L.oracle_openblas_open(openblas_candidates().encode()) != 0:
            raise RuntimeError("no OpenBLAS found among: " + openblas_candidates())
        self.name = L.oracle_openblas_name().decode()
        self.L = L

    def gemm(self, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, order=COLMAJOR):
        ta, tb = TRANS_OF[transa], TRANS_OF[transb]
        if C.dtype == np.complex64:
            al = np.array([complex(alpha).real, complex(alpha).imag], dtype=np.float32)
            be = np.array([complex(beta).real, complex(beta).imag], dtype=np.float32)
            self.L.oracle_openblas_cgemm(order, ta, tb, M, N, K, _ptr(al), _ptr(A), lda, _ptr(B), ldb, _ptr(be),
                                         _ptr(C), ldc)
            return C
        if C.dtype == np.float64:
            self.L.oracle_openblas_dgemm(order, ta, tb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C), ldc)
        elif C.dtype == np.float32:
            self.L.oracle_openblas_sgemm(order, ta, tb, M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C), ldc)
        else:
            al = np.array([complex(alpha).real, complex(alpha).imag])
            be = np.array([complex(beta).real, complex(beta).imag])
            self.L.oracle_openblas_zgemm(order, ta, tb, M, N, K, _ptr(al), _ptr(A), lda, _ptr(B), ldb, _ptr(be), _ptr(C), ldc)
        return C


class Reference:
    """The reference library (oracle/_ref/libblasx_ref.so), CPU path only.

    Calls with every dimension <= 1000 (<= 500 for Z) dispatch to the CPU BLAS
    the reference was compiled against (blas/dgemm.c:61-75); larger calls
    would take its cuBLAS path, which this class never uses.
    """

    def __init__(self):
        if not os.path.exists(REF_PATH):
            raise FileNotFoundError(REF_PATH)
        _preload_gfortran(os.path.join(_site(), "opencv_python_headless.libs"))
        L = ctypes.CDLL(REF_PATH)
        L.cblas_dgemm.argtypes = [_I] * 6 + [_D, _P, _I, _P, _I, _D, _P, _I]
        L.cblas_sgemm.argtypes = [_I] * 6 + [_F, _P, _I, _P, _I, _F, _P, _I]
        L.cblas_zgemm.argtypes = [_I] * 6 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.cblas_cgemm.argtypes = [_I] * 6 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.dgemm_.argtypes = [_P] * 13
        self.L = L

    def gemm(self, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, order=COLMAJOR,
             ta=None, tb=None):
        ta = TRANS_OF[transa] if ta is None else ta
        tb = TRANS_OF[transb] if tb is None else tb
        Ap = _ptr(A) if A is not None else None
        Bp = _ptr(B) if B is not None else None
        if C.dtype == np.float64:
            self.L.cblas_dgemm(order, ta, tb, M, N, K, alpha, Ap, lda, Bp, ldb, beta, _ptr(C), ldc)
        elif C.dtype == np.float32:
            self.L.cblas_sgemm(order, ta, tb, M, N, K, alpha, Ap, lda, Bp, ldb, beta, _ptr(C), ldc)
        elif C.dtype == np.complex64:
            al = np.array([complex(alpha).real, complex(alpha).imag], dtype=np.float32)
            be = np.array([complex(beta).real, complex(beta).imag], dtype=np.float32)
            self.L.cblas_cgemm(order, ta, tb, M, N, K, _ptr(al), Ap, lda, Bp, ldb, _ptr(be), _ptr(C), ldc)
        else:
            al = np.array([complex(alpha).real, complex(alpha).imag])
            be = np.array([complex(beta).real, complex(beta).imag])
            self.L.cblas_zgemm(order, ta, tb, M, N, K, _ptr(al), Ap, lda, Bp, ldb, _ptr(be), _ptr(C), ldc)
        return C
