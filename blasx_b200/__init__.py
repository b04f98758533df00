"""blasx_b200 -- B200-native tiled GEMM runtime behind the BLASX C ABI.

The product is the shared library ``libblasx_b200.so`` built from ``csrc/``
(CUDA C++ for sm_100a). Its C ABI is declared in ``include/blasx_b200.h`` and
replaces the GEMM entry points of linnanwang/BLASX: ``cblas_sgemm``,
``cblas_dgemm``, ``cblas_zgemm`` (include/cblas.h:424/454/514) and the F77
wrappers ``sgemm_``, ``dgemm_``, ``zgemm_`` (blas/dgemm.c:131-154).

This module is the Python host mirror of that interface (ctypes, no torch in
the signatures): the same names, argument order and meaning, and the same
error behaviour (``xerbla_`` text on stdout, C untouched). It loads the
in-tree library and raises if it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libblasx_b200.so")
HEADER = os.path.join(ROOT, "include", "blasx_b200.h")

CblasRowMajor, CblasColMajor = 101, 102
CblasNoTrans, CblasTrans, CblasConjTrans = 111, 112, 113
TRANS = {"N": CblasNoTrans, "T": CblasTrans, "C": CblasConjTrans}

BLASX_OK, BLASX_ERR_ARG, BLASX_ERR_CUDA, BLASX_ERR_NOMEM = 0, 1, 2, 3
BLASX_ERR_NODEVICE, BLASX_ERR_TIMEOUT, BLASX_ERR_UNSUPPORTED, BLASX_ERR_CLOSED = 4, 5, 6, 7

MODE_AUTO, MODE_NATIVE, MODE_OZAKI = 0, 1, 2

_P, _I, _D, _F = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float
_lib = None


class TilePlanStats(ctypes.Structure):
    _fields_ = [("tiles_m", _I), ("tiles_n", _I), ("tiles_k", _I), ("slots", _I),
                ("steps", ctypes.c_longlong), ("tile_loads", ctypes.c_longlong),
                ("tile_hits", ctypes.c_longlong), ("evictions", ctypes.c_longlong),
                ("operand_h2d_bytes", _D), ("min_operand_h2d_bytes", _D)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("cache_hits", ctypes.c_longlong),
                ("cache_misses", ctypes.c_longlong), ("grouped_launches", ctypes.c_longlong),
                ("grouped_requests", ctypes.c_longlong), ("max_inflight_seen", _I), ("reserved", _I),
                ("p50_ms", _D), ("p99_ms", _D), ("mean_ms", _D), ("max_ms", _D),
                ("flops", _D), ("seconds", _D), ("tflops", _D),
                ("admit_seconds", _D), ("admit_max_ms", _D), ("memory_waits", ctypes.c_longlong),
                ("head_holds", ctypes.c_longlong), ("alloc_seconds", _D), ("copy_seconds", _D),
                ("compute_enqueue_seconds", _D), ("mean_copy_in_ms", _D), ("mean_compute_ms", _D),
                ("mean_copy_out_ms", _D)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class CallStats(ctypes.Structure):
    _fields_ = [("seconds", _D), ("h2d_bytes", _D), ("d2h_bytes", _D), ("cache_hits", _D),
                ("cache_misses", _D), ("evictions", _D), ("path", _I), ("moduli", _I),
                ("tile", _I), ("host_copy", _I)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


def build(verbose: bool = False) -> str:
    from . import _build
    return _build.build(verbose=verbose)


def lib() -> ctypes.CDLL:
    """The loaded libblasx_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m blasx_b200._build` "
                              "(the GEMM path has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        L.cblas_sgemm.argtypes = [_I] * 6 + [_F, _P, _I, _P, _I, _F, _P, _I]
        L.cblas_dgemm.argtypes = [_I] * 6 + [_D, _P, _I, _P, _I, _D, _P, _I]
        L.cblas_zgemm.argtypes = [_I] * 6 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.cblas_cgemm.argtypes = [_I] * 6 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.cblas_ssyrk.argtypes = [_I] * 5 + [_F, _P, _I, _F, _P, _I]
        L.cblas_dsyrk.argtypes = [_I] * 5 + [_D, _P, _I, _D, _P, _I]
        L.cblas_zsyrk.argtypes = [_I] * 5 + [_P, _P, _I, _P, _P, _I]
        L.cblas_ssyr2k.argtypes = [_I] * 5 + [_F, _P, _I, _P, _I, _F, _P, _I]
        L.cblas_dsyr2k.argtypes = [_I] * 5 + [_D, _P, _I, _P, _I, _D, _P, _I]
        L.cblas_zsyr2k.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.cblas_csyrk.argtypes = [_I] * 5 + [_P, _P, _I, _P, _P, _I]
        L.cblas_csyr2k.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _P, _P, _I]
        L.cblas_cherk.argtypes = [_I] * 5 + [_F, _P, _I, _F, _P, _I]
        L.cblas_zherk.argtypes = [_I] * 5 + [_D, _P, _I, _D, _P, _I]
        L.cblas_cher2k.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _F, _P, _I]
        L.cblas_zher2k.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _D, _P, _I]
        for f in ("ssyrk_", "dsyrk_", "zsyrk_", "csyrk_", "cherk_", "zherk_"):
            getattr(L, f).argtypes = [_P] * 10
        for f in ("ssyr2k_", "dsyr2k_", "zsyr2k_", "csyr2k_", "cher2k_", "zher2k_"):
            getattr(L, f).argtypes = [_P] * 12
        L.blasx_dsyrk_device.argtypes = [_I] * 4 + [_D, _P, _I, _D, _P, _I, _P]
        L.blasx_dtrsm_device.argtypes = [_I] * 6 + [_D, _P, _I, _P, _I, _P]
        L.blasx_dtrmm_device.argtypes = [_I] * 6 + [_D, _P, _I, _P, _I, _P]
        for t, sc in (("s", _F), ("d", _D), ("c", _P), ("z", _P)):
            for kind in ("symm", "hemm") if t in "cz" else ("symm",):
                getattr(L, f"cblas_{t}{kind}").argtypes = [_I] * 5 + [sc, _P, _I, _P, _I, sc, _P, _I]
                getattr(L, f"{t}{kind}_").argtypes = [_P] * 12
            for kind in ("trmm", "trsm"):
                getattr(L, f"cblas_{t}{kind}").argtypes = [_I] * 7 + [sc, _P, _I, _P, _I]
                getattr(L, f"{t}{kind}_").argtypes = [_P] * 11
        for f in ("sgemm_", "dgemm_", "cgemm_", "zgemm_"):
            getattr(L, f).argtypes = [_P] * 13
        L.xerbla_.argtypes = [ctypes.c_char_p, _P]
        L.blasx_last_status.restype = _I
        L.blasx_last_error.restype = ctypes.c_char_p
        L.blasx_set_dgemm_mode.argtypes = [_I]
        L.blasx_set_hbm_budget.argtypes = [ctypes.c_size_t]
        L.blasx_set_tile.argtypes = [_I]
        L.blasx_set_host_staging.argtypes = [_I]
        L.blasx_get_call_stats.argtypes = [ctypes.POINTER(CallStats)]
        L.blasx_dgemm_device.argtypes = [_I] * 5 + [_D, _P, _I, _P, _I, _D, _P, _I, _P]
        L.blasx_sgemm_device.argtypes = [_I] * 5 + [_F, _P, _I, _P, _I, _F, _P, _I, _P]
        L.blasx_zgemm_device.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _P, _P, _I, _P]
        L.blasx_cgemm_device.argtypes = [_I] * 5 + [_P, _P, _I, _P, _I, _P, _P, _I, _P]
        L.blasx_dgemm_device_noalloc.argtypes = [_I] * 5 + [_D, _P, _I, _P, _I, _D, _P, _I, _P]
        L.blasx_dgemm_device_noalloc_status.argtypes = [_P]
        L.blasx_test_stall_residue_gemm.argtypes = [_I, ctypes.c_longlong]
        L.blasx_test_fail_allocation.argtypes = [_I]
        L.blasx_kernel_launch_count.restype = ctypes.c_uint64
        L.blasx_tile_plan.argtypes = [ctypes.c_longlong] * 5 + [_I, _I, ctypes.POINTER(TilePlanStats)]
        L.blasx_serve_start.argtypes = [ctypes.c_size_t, ctypes.c_size_t, _I]
        L.blasx_serve_invalidate.argtypes = [_P]
        L.blasx_serve_get_stats.argtypes = [ctypes.POINTER(ServeStats)]
        L.blasx_profile_enable.argtypes = [_I]
        L.blasx_profile_read.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long), _I]
        _lib = L
    return _lib


def kernel_launch_count() -> int:
    """Kernels launched by the library so far (all threads)."""
    return int(lib().blasx_kernel_launch_count())


def declared_symbols() -> list[str]:
    """Function names declared in include/blasx_b200.h (the C ABI)."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M)
    return sorted({n for n in names if not n.startswith("__")})


def _addr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    raise TypeError(f"cannot take the address of {type(x)}")


def _cpair(v) -> np.ndarray:
    v = complex(v)
    return np.array([v.real, v.imag], dtype=np.float64)


# ---------------------------------------------------------------------------
# CBLAS mirror (include/cblas.h:424/454/514)
# ---------------------------------------------------------------------------

def cblas_sgemm(Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    lib().cblas_sgemm(Order, TransA, TransB, M, N, K, alpha, _addr(A), lda, _addr(B), ldb, beta,
                      _addr(C), ldc)


def cblas_dgemm(Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    lib().cblas_dgemm(Order, TransA, TransB, M, N, K, alpha, _addr(A), lda, _addr(B), ldb, beta,
                      _addr(C), ldc)


def cblas_zgemm(Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    al, be = _cpair(alpha), _cpair(beta)
    lib().cblas_zgemm(Order, TransA, TransB, M, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb,
                      be.ctypes.data, _addr(C), ldc)


UPLO = {"U": 121, "L": 122}
CblasUpper, CblasLower = 121, 122


def cblas_ssyrk(Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc):
    lib().cblas_ssyrk(Order, Uplo, Trans, N, K, alpha, _addr(A), lda, beta, _addr(C), ldc)


def cblas_dsyrk(Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc):
    lib().cblas_dsyrk(Order, Uplo, Trans, N, K, alpha, _addr(A), lda, beta, _addr(C), ldc)


def cblas_zsyrk(Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc):
    al, be = _cpair(alpha), _cpair(beta)
    lib().cblas_zsyrk(Order, Uplo, Trans, N, K, al.ctypes.data, _addr(A), lda, be.ctypes.data, _addr(C), ldc)


def cblas_ssyr2k(Order, Uplo, Trans, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    lib().cblas_ssyr2k(Order, Uplo, Trans, N, K, alpha, _addr(A), lda, _addr(B), ldb, beta, _addr(C), ldc)


def cblas_dsyr2k(Order, Uplo, Trans, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    lib().cblas_dsyr2k(Order, Uplo, Trans, N, K, alpha, _addr(A), lda, _addr(B), ldb, beta, _addr(C), ldc)


def cblas_zsyr2k(Order, Uplo, Trans, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    al, be = _cpair(alpha), _cpair(beta)
    lib().cblas_zsyr2k(Order, Uplo, Trans, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb,
                       be.ctypes.data, _addr(C), ldc)


def _f77_syr(fn, ctype, uplo, trans, n, k, alpha, A, lda, beta, C, ldc, B=None, ldb=None, cplx=False,
             pair=None):
    u = ctypes.c_char(uplo.encode() if isinstance(uplo, str) else uplo)
    t = ctypes.c_char(trans.encode() if isinstance(trans, str) else trans)
    ints = [ctypes.c_int(v) for v in (n, k, lda, ldc, ldb or 1)]
    if cplx:
        al, be = (pair or _cpair)(alpha), (pair or _cpair)(beta)
        pa, pb = al.ctypes.data, be.ctypes.data
    else:
        al, be = ctype(alpha), ctype(beta)
        pa, pb = ctypes.addressof(al), ctypes.addressof(be)
    r = ctypes.byref
    if B is None:
        fn(r(u), r(t), r(ints[0]), r(ints[1]), pa, _addr(A), r(ints[2]), pb, _addr(C), r(ints[3]))
    else:
        fn(r(u), r(t), r(ints[0]), r(ints[1]), pa, _addr(A), r(ints[2]), _addr(B), r(ints[4]), pb, _addr(C),
           r(ints[3]))


def ssyrk_(uplo, trans, n, k, alpha, A, lda, beta, C, ldc):
    _f77_syr(lib().ssyrk_, ctypes.c_float, uplo, trans, n, k, alpha, A, lda, beta, C, ldc)


def dsyrk_(uplo, trans, n, k, alpha, A, lda, beta, C, ldc):
    _f77_syr(lib().dsyrk_, ctypes.c_double, uplo, trans, n, k, alpha, A, lda, beta, C, ldc)


def zsyrk_(uplo, trans, n, k, alpha, A, lda, beta, C, ldc):
    _f77_syr(lib().zsyrk_, None, uplo, trans, n, k, alpha, A, lda, beta, C, ldc, cplx=True)


def cblas_csyrk(Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc):
    al, be = _cpair32(alpha), _cpair32(beta)
    lib().cblas_csyrk(Order, Uplo, Trans, N, K, al.ctypes.data, _addr(A), lda, be.ctypes.data, _addr(C), ldc)


def cblas_csyr2k(Order, Uplo, Trans, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    al, be = _cpair32(alpha), _cpair32(beta)
    lib().cblas_csyr2k(Order, Uplo, Trans, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb, be.ctypes.data,
                       _addr(C), ldc)


def cblas_cherk(Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc):
    lib().cblas_cherk(Order, Uplo, Trans, N, K, float(alpha), _addr(A), lda, float(beta), _addr(C), ldc)


def cblas_zherk(Order, Uplo, Trans, N, K, alpha, A, lda, beta, C, ldc):
    lib().cblas_zherk(Order, Uplo, Trans, N, K, float(alpha), _addr(A), lda, float(beta), _addr(C), ldc)


def cblas_cher2k(Order, Uplo, Trans, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    al = _cpair32(alpha)
    lib().cblas_cher2k(Order, Uplo, Trans, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb, float(beta),
                       _addr(C), ldc)


def cblas_zher2k(Order, Uplo, Trans, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    al = _cpair(alpha)
    lib().cblas_zher2k(Order, Uplo, Trans, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb, float(beta),
                       _addr(C), ldc)


def _f77_her(fn, ctype, uplo, trans, n, k, alpha, A, lda, beta, C, ldc, B=None, ldb=None, pair=None):
    """F77 HERK / HER2K: real beta (and real HERK alpha) by pointer; HER2K's
    complex alpha as an (re, im) pair of `pair` (_cpair32 or _cpair)."""
    u, t = _char(uplo), _char(trans)
    ints = [ctypes.c_int(v) for v in (n, k, lda, ldc, ldb or 1)]
    be = ctype(beta)
    if pair is None:
        al = ctype(alpha)
        pa = ctypes.addressof(al)
    else:
        al = pair(alpha)
        pa = al.ctypes.data
    r = ctypes.byref
    if B is None:
        fn(r(u), r(t), r(ints[0]), r(ints[1]), pa, _addr(A), r(ints[2]), r(be), _addr(C), r(ints[3]))
    else:
        fn(r(u), r(t), r(ints[0]), r(ints[1]), pa, _addr(A), r(ints[2]), _addr(B), r(ints[4]), r(be), _addr(C),
           r(ints[3]))


def cherk_(uplo, trans, n, k, alpha, A, lda, beta, C, ldc):
    _f77_her(lib().cherk_, ctypes.c_float, uplo, trans, n, k, alpha, A, lda, beta, C, ldc)


def zherk_(uplo, trans, n, k, alpha, A, lda, beta, C, ldc):
    _f77_her(lib().zherk_, ctypes.c_double, uplo, trans, n, k, alpha, A, lda, beta, C, ldc)


def cher2k_(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    _f77_her(lib().cher2k_, ctypes.c_float, uplo, trans, n, k, alpha, A, lda, beta, C, ldc, B=B, ldb=ldb,
             pair=_cpair32)


def zher2k_(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    _f77_her(lib().zher2k_, ctypes.c_double, uplo, trans, n, k, alpha, A, lda, beta, C, ldc, B=B, ldb=ldb,
             pair=_cpair)


def csyrk_(uplo, trans, n, k, alpha, A, lda, beta, C, ldc):
    _f77_syr(lib().csyrk_, None, uplo, trans, n, k, alpha, A, lda, beta, C, ldc, cplx=True, pair=_cpair32)


def dsyr2k_(uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    _f77_syr(lib().dsyr2k_, ctypes.c_double, uplo, trans, n, k, alpha, A, lda, beta, C, ldc, B=B, ldb=ldb)


def dsyrk_device(uplo, trans, N, K, alpha, A, lda, beta, C, ldc, stream=None):
    """Device-resident DSYRK on device pointers (ints or tensors with data_ptr)."""
    s = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else _addr(stream))
    u = UPLO[uplo] if isinstance(uplo, str) else uplo
    t = TRANS[trans] if isinstance(trans, str) else trans
    return lib().blasx_dsyrk_device(u, t, N, K, alpha, _addr(A), lda, beta, _addr(C), ldc, s)


def dtrsm_device(side, uplo, trans, diag, M, N, alpha, A, lda, B, ldb, stream=None):
    """Device-resident DTRSM on device pointers (ints or tensors with data_ptr)."""
    s = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else _addr(stream))
    args = [SIDE.get(side, side), UPLO.get(uplo, uplo), TRANS.get(trans, trans), DIAG.get(diag, diag)]
    return lib().blasx_dtrsm_device(*args, M, N, alpha, _addr(A), lda, _addr(B), ldb, s)


def dtrmm_device(side, uplo, trans, diag, M, N, alpha, A, lda, B, ldb, stream=None):
    """Device-resident DTRMM on device pointers (ints or tensors with data_ptr)."""
    s = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else _addr(stream))
    args = [SIDE.get(side, side), UPLO.get(uplo, uplo), TRANS.get(trans, trans), DIAG.get(diag, diag)]
    return lib().blasx_dtrmm_device(*args, M, N, alpha, _addr(A), lda, _addr(B), ldb, s)


def _cpair32(v) -> np.ndarray:
    v = complex(v)
    return np.array([v.real, v.imag], dtype=np.float32)


def cblas_cgemm(Order, TransA, TransB, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    al, be = _cpair32(alpha), _cpair32(beta)
    lib().cblas_cgemm(Order, TransA, TransB, M, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb,
                      be.ctypes.data, _addr(C), ldc)


def cgemm_(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    ta = ctypes.c_char(transa.encode() if isinstance(transa, str) else transa)
    tb = ctypes.c_char(transb.encode() if isinstance(transb, str) else transb)
    ints = [ctypes.c_int(v) for v in (m, n, k, lda, ldb, ldc)]
    al, be = _cpair32(alpha), _cpair32(beta)
    r = ctypes.byref
    lib().cgemm_(r(ta), r(tb), r(ints[0]), r(ints[1]), r(ints[2]), al.ctypes.data, _addr(A), r(ints[3]),
                 _addr(B), r(ints[4]), be.ctypes.data, _addr(C), r(ints[5]))


SIDE = {"L": 141, "R": 142}
DIAG = {"N": 131, "U": 132}
CblasLeft, CblasRight = 141, 142
CblasNonUnit, CblasUnit = 131, 132


def _scalar_value(tag, v):
    """A cblas_ scalar: by value for s / d, the address of an (re, im) pair
    for c / z. The second item keeps the pair alive for the call."""
    if tag in "sd":
        return v, None
    pair = _cpair32(v) if tag == "c" else _cpair(v)
    return pair.ctypes.data, pair


def _scalar_ref(tag, v):
    """An F77 scalar: always by address."""
    if tag in "sd":
        box = (ctypes.c_float if tag == "s" else ctypes.c_double)(v)
        return ctypes.addressof(box), box
    pair = _cpair32(v) if tag == "c" else _cpair(v)
    return pair.ctypes.data, pair


def _char(c):
    return ctypes.c_char(c.encode() if isinstance(c, str) else c)


def _symm_fn(tag, kind):
    name = f"cblas_{tag}{kind}"

    def call(Order, Side, Uplo, M, N, alpha, A, lda, B, ldb, beta, C, ldc):
        al, keep_a = _scalar_value(tag, alpha)
        be, keep_b = _scalar_value(tag, beta)
        getattr(lib(), name)(Order, Side, Uplo, M, N, al, _addr(A), lda, _addr(B), ldb, be, _addr(C), ldc)

    call.__name__ = call.__qualname__ = name
    return call


def _trmm_fn(tag, kind="trmm"):
    name = f"cblas_{tag}{kind}"

    def call(Order, Side, Uplo, TransA, Diag, M, N, alpha, A, lda, B, ldb):
        al, keep = _scalar_value(tag, alpha)
        getattr(lib(), name)(Order, Side, Uplo, TransA, Diag, M, N, al, _addr(A), lda, _addr(B), ldb)

    call.__name__ = call.__qualname__ = name
    return call


def _symm_f77(tag, kind):
    name = f"{tag}{kind}_"

    def call(side, uplo, m, n, alpha, A, lda, B, ldb, beta, C, ldc):
        sd, up = _char(side), _char(uplo)
        ints = [ctypes.c_int(v) for v in (m, n, lda, ldb, ldc)]
        pa, keep_a = _scalar_ref(tag, alpha)
        pb, keep_b = _scalar_ref(tag, beta)
        r = ctypes.byref
        getattr(lib(), name)(r(sd), r(up), r(ints[0]), r(ints[1]), pa, _addr(A), r(ints[2]), _addr(B),
                             r(ints[3]), pb, _addr(C), r(ints[4]))

    call.__name__ = call.__qualname__ = name
    return call


def _trmm_f77(tag, kind="trmm"):
    name = f"{tag}{kind}_"

    def call(side, uplo, transa, diag, m, n, alpha, A, lda, B, ldb):
        chars = [_char(c) for c in (side, uplo, transa, diag)]
        ints = [ctypes.c_int(v) for v in (m, n, lda, ldb)]
        pa, keep = _scalar_ref(tag, alpha)
        r = ctypes.byref
        getattr(lib(), name)(*(r(c) for c in chars), r(ints[0]), r(ints[1]), pa, _addr(A), r(ints[2]),
                             _addr(B), r(ints[3]))

    call.__name__ = call.__qualname__ = name
    return call


# cblas_?symm / ?hemm / ?trmm / ?trsm and their F77 forms (blas/dsymm.c,
# blas/zhemm.c, blas/dtrmm.c, blas/dtrsm.c in the reference): same argument
# order and meaning.
cblas_ssymm, cblas_dsymm = _symm_fn("s", "symm"), _symm_fn("d", "symm")
cblas_csymm, cblas_zsymm = _symm_fn("c", "symm"), _symm_fn("z", "symm")
cblas_chemm, cblas_zhemm = _symm_fn("c", "hemm"), _symm_fn("z", "hemm")
cblas_strmm, cblas_dtrmm, cblas_ctrmm, cblas_ztrmm = (_trmm_fn(t) for t in "sdcz")
ssymm_, dsymm_, csymm_, zsymm_ = (_symm_f77(t, "symm") for t in "sdcz")
chemm_, zhemm_ = _symm_f77("c", "hemm"), _symm_f77("z", "hemm")
strmm_, dtrmm_, ctrmm_, ztrmm_ = (_trmm_f77(t) for t in "sdcz")
cblas_strsm, cblas_dtrsm, cblas_ctrsm, cblas_ztrsm = (_trmm_fn(t, "trsm") for t in "sdcz")
strsm_, dtrsm_, ctrsm_, ztrsm_ = (_trmm_f77(t, "trsm") for t in "sdcz")


def _f77(fn, ctype, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, cplx=False):
    ta = ctypes.c_char(transa.encode() if isinstance(transa, str) else transa)
    tb = ctypes.c_char(transb.encode() if isinstance(transb, str) else transb)
    ints = [ctypes.c_int(v) for v in (m, n, k, lda, ldb, ldc)]
    if cplx:
        al, be = _cpair(alpha), _cpair(beta)
        pa, pb = al.ctypes.data, be.ctypes.data
    else:
        al, be = ctype(alpha), ctype(beta)
        pa, pb = ctypes.addressof(al), ctypes.addressof(be)
    r = ctypes.byref
    fn(r(ta), r(tb), r(ints[0]), r(ints[1]), r(ints[2]), pa, _addr(A), r(ints[3]), _addr(B),
       r(ints[4]), pb, _addr(C), r(ints[5]))


def sgemm_(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    _f77(lib().sgemm_, ctypes.c_float, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)


def dgemm_(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    _f77(lib().dgemm_, ctypes.c_double, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)


def zgemm_(transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    _f77(lib().zgemm_, None, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, cplx=True)


def gemm(transa, transb, alpha, A, B, beta, C):
    """C <- alpha op(A) op(B) + beta C on Fortran-ordered numpy arrays."""
    M, N = C.shape
    K = A.shape[1] if transa == "N" else A.shape[0]
    args = (CblasColMajor, TRANS[transa], TRANS[transb], M, N, K, alpha, A, max(1, A.shape[0]),
            B, max(1, B.shape[0]), beta, C, max(1, M))
    {np.float32: cblas_sgemm, np.float64: cblas_dgemm, np.complex64: cblas_cgemm,
     np.complex128: cblas_zgemm}[C.dtype.type](*args)
    return C


# ---------------------------------------------------------------------------
# extensions
# ---------------------------------------------------------------------------

def gemm_device(transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, stream=None,
                dtype="d"):
    """Device-resident GEMM on device pointers (ints or tensors with data_ptr)."""
    L = lib()
    s = _addr(stream) if stream is not None and not hasattr(stream, "cuda_stream") else \
        (stream.cuda_stream if stream is not None else None)
    ta = TRANS[transa] if isinstance(transa, str) else transa
    tb = TRANS[transb] if isinstance(transb, str) else transb
    if dtype == "d":
        return L.blasx_dgemm_device(ta, tb, M, N, K, alpha, _addr(A), lda, _addr(B), ldb, beta, _addr(C), ldc, s)
    if dtype == "s":
        return L.blasx_sgemm_device(ta, tb, M, N, K, alpha, _addr(A), lda, _addr(B), ldb, beta, _addr(C), ldc, s)
    if dtype == "c":
        al, be = _cpair32(alpha), _cpair32(beta)
        return L.blasx_cgemm_device(ta, tb, M, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb,
                                    be.ctypes.data, _addr(C), ldc, s)
    al, be = _cpair(alpha), _cpair(beta)
    return L.blasx_zgemm_device(ta, tb, M, N, K, al.ctypes.data, _addr(A), lda, _addr(B), ldb,
                                be.ctypes.data, _addr(C), ldc, s)


def last_status() -> int:
    return lib().blasx_last_status()


def last_error() -> str:
    return lib().blasx_last_error().decode()


def call_stats() -> dict:
    s = CallStats()
    lib().blasx_get_call_stats(ctypes.byref(s))
    return s.as_dict()


def set_dgemm_mode(mode: int) -> int:
    return lib().blasx_set_dgemm_mode(mode)


def set_hbm_budget(nbytes: int) -> int:
    return lib().blasx_set_hbm_budget(nbytes)


def set_tile(tile: int) -> int:
    return lib().blasx_set_tile(tile)


def set_host_staging(on: bool) -> int:
    """Pageable host operands: staged through pinned bounce buffers (True,
    the default) or registered for the call (False). Returns the previous
    setting."""
    return lib().blasx_set_host_staging(1 if on else 0)


def finalize() -> int:
    return lib().blasx_finalize()


def serve_start(hbm_budget: int = 0, cache_bytes: int = 0, max_inflight: int = 0) -> int:
    """Route host GEMM calls of all threads through the serving loop."""
    return lib().blasx_serve_start(hbm_budget, cache_bytes, max_inflight)


def serve_stop() -> int:
    return lib().blasx_serve_stop()


def test_stall_residue_gemm(launches: int, wait_cycles: int) -> int:
    """Test hook: the next `launches` residue-GEMM launches stall one stage of
    CTA 0 and give up after `wait_cycles` (the call reports BLASX_ERR_TIMEOUT)."""
    return lib().blasx_test_stall_residue_gemm(launches, wait_cycles)


def test_fail_allocation(nth: int) -> int:
    """Test hook: the nth device allocation from now on fails (0 disarms)."""
    return lib().blasx_test_fail_allocation(nth)


def serve_invalidate(host_buffer) -> int:
    """Drop cached device copies of an operand modified in place."""
    return lib().blasx_serve_invalidate(_addr(host_buffer))


def serve_stats() -> dict:
    s = ServeStats()
    lib().blasx_serve_get_stats(ctypes.byref(s))
    return s.as_dict()


def serve_reset_stats() -> int:
    return lib().blasx_serve_reset_stats()


POLICY_BELADY, POLICY_LRU = 0, 1


def tile_plan(M, N, K, tile, budget_bytes, elem_bytes=8, policy=POLICY_BELADY) -> dict:
    """Host-only schedule of an out-of-core GEMM (no GPU needed)."""
    s = TilePlanStats()
    rc = lib().blasx_tile_plan(M, N, K, tile, budget_bytes, elem_bytes, policy, ctypes.byref(s))
    if rc != 0:
        raise ValueError(f"blasx_tile_plan failed ({rc})")
    return s.as_dict()


PHASES = ("slice", "residue_gemm", "reconstruct", "native")


def profile_enable(on: bool = True) -> bool:
    """Turn per-phase CUDA-event timing on/off (resets the totals)."""
    return bool(lib().blasx_profile_enable(1 if on else 0))


def profile_read() -> dict:
    """Per-phase device time (ms) and span counts since profile_enable."""
    ms = (ctypes.c_double * 4)()
    cnt = (ctypes.c_long * 4)()
    lib().blasx_profile_read(ms, cnt, 4)
    return {p: {"ms": ms[i], "count": cnt[i]} for i, p in enumerate(PHASES)}
