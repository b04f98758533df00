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


# ---- the device's FP64-limb reconstruction, restated ---------------------------
# The reconstruction kernel (blasx_b200/csrc/ozaki_dev.cuh: crt_sums4 and
# crt_round) turns the unsigned residues u_l = X mod m_l of an entry into
# RN(X) without integer arithmetic: 40-bit limbs of the CRT weights, exact
# FP64 limb sums, the quotient by M, the exact limb differences, and a
# correctly rounded sum of three doubles by rounding to odd (Boldo and
# Melquiond, IEEE Trans. Computers 57(4), 2008). Every product and sum below
# is exact by the bounds the kernel's comments state, so plain Python float
# arithmetic (round to nearest) reproduces the kernel's fused multiply-adds
# bit for bit; ``fp_limb_tables`` asserts those bounds.

FP_CRT_MAX = 17  # moduli the FP64-limb method serves (M < 2^133)


def fp_limbs(n: int) -> int:
    return 2 if n <= 10 else 3 if n <= 15 else 4


def _limb40(v: int, k: int) -> int:
    return ((v >> (40 * k)) & ((1 << 40) - 1)) << (40 * k)


def fp_limb_tables(n: int):
    """(moduli, M, wq, cq, M40, invM) as the kernel's constant tables hold
    them: wq[l][k] = limb k of weight l times 2^8, cq[k] = sum_l wq[l][k],
    M40[k] = limb k of M."""
    assert n <= FP_CRT_MAX
    ms, M, w, _ = crt(n)
    L = fp_limbs(n)
    assert M < 2 ** (40 * L) and M < 2 ** 133
    wq = [[float(_limb40(wl, k) << 8) for k in range(L)] for wl in w]
    cq = [float(sum(_limb40(wl, k) << 8 for wl in w)) for k in range(L)]
    M40 = [float(_limb40(M, k)) for k in range(L)]
    for k in range(L):
        assert int(cq[k]) == sum(_limb40(wl, k) << 8 for wl in w)  # exact
        assert all(int(wq[l][k]) == _limb40(w[l], k) << 8 for l in range(n))
        assert int(M40[k]) == _limb40(M, k)
        # every partial limb sum lies in (-cq, S_k] and S_k < n 255 2^(40k+40)
        assert cq[k] < 2.0 ** (40 * k + 53) and n * 255 * 2.0 ** (40 * k + 40) < 2.0 ** (40 * k + 53)
    return ms, M, wq, cq, M40, 1.0 / float(M)


def _two_sum(a: float, b: float):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def _add_round_odd(a: float, b: float) -> float:
    s, e = _two_sum(a, b)
    if e != 0.0:
        bits = int(np.float64(s).view(np.int64))
        if not bits & 1:
            bits += 1 if (e > 0.0) == (s > 0.0) else -1
            s = float(np.int64(bits).view(np.float64))
    return s


def crt_fp64(u, tables) -> float:
    """RN(X) for the residues u_l = X mod m_l (|X| < M / 4), as the kernel
    computes it."""
    ms, M, wq, cq, M40, invM = tables
    L = len(cq)
    S = [-c for c in cq]
    for l, ul in enumerate(u):
        d = 1.0 + ul / 256.0  # the bit pattern 0x3FF00000 | u << 12 in the high word
        for k in range(L):
            S[k] = d * wq[l][k] + S[k]
    q = float(round((S[L - 1] + S[L - 2]) * invM))
    D = [S[k] - q * M40[k] for k in range(L)]
    if L == 2:
        x = D[1] + D[0]
    else:
        top = D[3] + D[2] if L == 4 else D[2]
        uh, ul = _two_sum(D[1], D[0])
        th, tl = _two_sum(top, uh)
        x = th + _add_round_odd(tl, ul)
    return x + 0.0


# ---- the device's residue computation, restated --------------------------------
# The slicing kernels (blasx_b200/csrc/ozaki_dev.cuh: residue_s) take the
# symmetric residue of a scaled integer v (|v| < 2^62) for an odd modulus m
# from the eight bytes b_k of the biased value v + 2^62: two byte dot products
# against the constants 2^(8k) mod m plus -2^62 mod m give s = v (mod m); with
# h = (m - 1) / 2 and t = s + h < 2^20, the quotient q of t by m is the high
# word of s * ceil(2^32 / m) + h * ceil(2^32 / m), and s - q m lies in [-h, h].
# For m = 256 the residue is the low byte of v.

def residue_bytes(v: int, m: int) -> int:
    a = v + (1 << 62)
    if m == 256:
        b = a & 255
        return b - 256 if b >= 128 else b
    h = (m - 1) // 2
    s = sum(((a >> (8 * k)) & 255) * ((1 << (8 * k)) % m) for k in range(8))
    s += (m - (1 << 62) % m) % m
    assert s + h < (1 << 20)
    magic = ((1 << 32) + m - 1) // m
    q = (s * magic + h * magic) >> 32
    assert q == (s + h) // m
    return s - q * m
