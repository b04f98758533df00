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
