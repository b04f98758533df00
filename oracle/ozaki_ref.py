"""CPU restatement of the emulated (Ozaki scheme II) GEMM -- TEST
INFRASTRUCTURE ONLY (used by tests/ to check the method and to calibrate the
modulus-count estimate; never by the shipped library).

Method: Ozaki, Uchino, Imamura, "Ozaki Scheme II: A GEMM-oriented emulation
of floating-point matrix multiplication using an integer modular technique"
(2025). Restated with exact Python integers:

1. each row of A / column of B is scaled by a power of two and rounded to an
   integer, |a'| < 2^P and ||a'_i||_2 < 2^Q, so every scaled dot product is
   below M / 4 (M = product of the moduli);
2. symmetric residues of the scaled integers for each modulus;
3. one integer GEMM per modulus, reduced mod m;
4. the Chinese remainder theorem recovers the exact scaled product, which is
   unscaled to floating point.

The result of step 4 must equal the exact integer product of the scaled
operands: the check ``emulate(..., verify=True)`` asserts it.
"""
from __future__ import annotations

import math

import numpy as np

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
          223, 217, 211, 199, 197, 193, 191, 181, 179, 173]


def crt(n: int):
    """(moduli, M, weights, Q) for the first n moduli; Q: 2^(2Q) <= M/4."""
    ms = MODULI[:n]
    M = math.prod(ms)
    w = [(M // m) * pow((M // m) % m, -1, m) for m in ms]
    Q = int(math.floor((math.log2(M) - 2) / 2))
    return ms, M, w, Q


def _sym(x: int, m: int) -> int:
    r = x % m
    return r - m if r > (m - 1) // 2 else r


def _ilogb(x: float) -> int:
    return math.frexp(x)[1] - 1


def exponents(X: np.ndarray, axis: int, Q: int, P: int = 62) -> np.ndarray:
    """Per-row (axis=1) or per-column (axis=0) exponents e with
    2^e ||x||_2 < 2^Q and 2^e max|x| < 2^P (0 for an all-zero line)."""
    amax = np.max(np.abs(X), axis=axis)
    n2 = np.sqrt(np.sum(X * X, axis=axis))
    out = np.zeros(amax.shape, dtype=np.int64)
    for t in range(amax.size):
        if amax[t] > 0:
            out[t] = min(Q - 1 - _ilogb(float(n2[t])), P - 1 - _ilogb(float(amax[t])))
    return out


def emulate(A: np.ndarray, B: np.ndarray, n: int, P: int = 62, verify: bool = False):
    """Emulated op(A) @ op(B) for float64 A (M x K), B (K x N) with n moduli.

    Returns (C, Q). With verify=True asserts that the CRT reconstruction is
    the exact integer product of the scaled operands.
    """
    ms, M, w, Q = crt(n)
    ea = exponents(A, 1, Q, P)
    eb = exponents(B, 0, Q, P)
    Ai = [[int(round(math.ldexp(float(A[i, k]), int(ea[i])))) for k in range(A.shape[1])]
          for i in range(A.shape[0])]
    Bi = [[int(round(math.ldexp(float(B[k, j]), int(eb[j])))) for j in range(B.shape[1])]
          for k in range(B.shape[0])]
    rows, cols, K = A.shape[0], B.shape[1], A.shape[1]
    U = []
    for m in ms:
        ra = np.array([[_sym(x, m) for x in r] for r in Ai], dtype=np.int64)
        rb = np.array([[_sym(x, m) for x in r] for r in Bi], dtype=np.int64)
        U.append((ra @ rb) % m)  # exact: |residue| <= 128, K small
    C = np.empty((rows, cols), dtype=np.float64)
    for i in range(rows):
        for j in range(cols):
            x = sum(int(U[l][i, j]) * w[l] for l in range(n)) % M
            if 2 * x >= M:
                x -= M
            if verify:
                exact = sum(Ai[i][k] * Bi[k][j] for k in range(K))
                assert x == exact, (i, j)
            C[i, j] = math.ldexp(float(x), -int(ea[i]) - int(eb[j])) if x else 0.0
    return C, Q
