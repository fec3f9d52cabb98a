"""Python access to libmublis (B200 build) through its C ABI.

The library is the product; this module only loads it and declares the
signatures of its exported entry points, the way the reference's
``test/correctness/check_cblas.py:57-139`` binds the reference build:

* ``cblas_{s,d}{gemm,symm,syrk,syr2k,trmm,trsm}`` (``include/cblas.h``),
* ``mublis_{s,d}*`` and ``mublis_l3_{s,d}driver`` (``include/mublis.h``),
* ``mublis_b200_*`` extensions (``include/mublis_b200.h``).

There is no fallback: if ``lib/libmublis.so`` has not been built, ``load()``
raises.  Every routine returns an ``int`` status (``mublis_*``) or reports
through ``cblas_xerbla`` (``cblas_*``), as in the reference.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR / "lib" / "libmublis.so"

# CBLAS enums (include/cblas.h)
ROW, COL = 101, 102
NO_TRANS, TRANS = 111, 112
UPPER, LOWER = 121, 122
NON_UNIT, UNIT = 131, 132
LEFT, RIGHT = 141, 142

# MuBLIS enums (include/mublis.h)
M_NO_TRANSPOSE, M_TRANSPOSE = 0, 1
M_DENSE, M_LOWER, M_UPPER = 0, 1, 2
M_LEFT, M_RIGHT = 0, 1
M_NON_UNIT, M_UNIT = 0, 1
STRUC_GENERAL, STRUC_SYMMETRIC, STRUC_TRIANGULAR = 0, 1, 2
DIAG_NONUNIT, DIAG_UNIT, DIAG_INVERT = 0, 1, 2
L3_ALL, L3_LOWER, L3_UPPER = 0, 1, 2


class Operand(ctypes.Structure):
    _fields_ = [("struc", ctypes.c_int), ("uplo", ctypes.c_int), ("diag", ctypes.c_int)]


class Domain(ctypes.Structure):
    _fields_ = [("jp", ctypes.c_int), ("ji", ctypes.c_int), ("pi", ctypes.c_int)]


class Product(ctypes.Structure):
    _fields_ = [("domain", Domain), ("a", Operand), ("b", Operand)]


_I, _P, _L, _U32 = ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_uint32


class GemmProblem(ctypes.Structure):
    """mublis_b200_gemm_problem_t (include/mublis_b200.h)."""
    _fields_ = [("trans_a", ctypes.c_int), ("trans_b", ctypes.c_int), ("m", ctypes.c_int),
                ("n", ctypes.c_int), ("k", ctypes.c_int), ("alpha", ctypes.c_double),
                ("beta", ctypes.c_double), ("a", ctypes.c_void_p), ("lda", ctypes.c_int),
                ("b", ctypes.c_void_p), ("ldb", ctypes.c_int), ("c", ctypes.c_void_p),
                ("ldc", ctypes.c_int)]


class TrsmProblem(ctypes.Structure):
    """mublis_b200_trsm_problem_t."""
    _fields_ = [("uplo", ctypes.c_int), ("trans_a", ctypes.c_int), ("diag", ctypes.c_int),
                ("m", ctypes.c_int), ("n", ctypes.c_int), ("alpha", ctypes.c_double),
                ("a", ctypes.c_void_p), ("lda", ctypes.c_int), ("b", ctypes.c_void_p),
                ("ldb", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    """mublis_b200_server_config_t."""
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("streams", ctypes.c_int),
                ("batch_window_us", ctypes.c_int), ("small_max_dim", ctypes.c_int),
                ("max_batch", ctypes.c_int), ("sform", ctypes.c_char_p),
                ("dform", ctypes.c_char_p)]


class ServerStats(ctypes.Structure):
    """mublis_b200_server_stats_t."""
    _fields_ = [("completed", ctypes.c_ulonglong), ("batches", ctypes.c_ulonglong),
                ("batched_requests", ctypes.c_ulonglong), ("queue_depth", ctypes.c_ulonglong),
                ("p50_latency_s", ctypes.c_double), ("p99_latency_s", ctypes.c_double),
                ("mean_latency_s", ctypes.c_double), ("tflops", ctypes.c_double),
                ("elapsed_s", ctypes.c_double), ("hbm_in_use", ctypes.c_size_t)]


# "scalar" is replaced by c_float / c_double per precision.
CBLAS_SIGNATURES = {
    "gemm": [_I, _I, _I, _I, _I, _I, "scalar", _P, _I, _P, _I, "scalar", _P, _I],
    "symm": [_I, _I, _I, _I, _I, "scalar", _P, _I, _P, _I, "scalar", _P, _I],
    "syrk": [_I, _I, _I, _I, _I, "scalar", _P, _I, "scalar", _P, _I],
    "syr2k": [_I, _I, _I, _I, _I, "scalar", _P, _I, _P, _I, "scalar", _P, _I],
    "trmm": [_I, _I, _I, _I, _I, _I, _I, "scalar", _P, _I, _P, _I],
    "trsm": [_I, _I, _I, _I, _I, _I, _I, "scalar", _P, _I, _P, _I],
}

MUBLIS_SIGNATURES = {
    "gemm": [_I, _I, _I, _I, _I, "scalar", _P, _I, _I, _P, _I, _I, "scalar", _P, _I, _I],
    "symm": [_I, _I, _I, _I, "scalar", _P, _I, _I, _P, _I, _I, "scalar", _P, _I, _I],
    "syrk": [_I, _I, _I, _I, "scalar", _P, _I, _I, "scalar", _P, _I, _I],
    "syr2k": [_I, _I, _I, _I, "scalar", _P, _I, _I, _P, _I, _I, "scalar", _P, _I, _I],
    "trmm": [_I, _I, _I, _I, _I, _I, "scalar", _P, _I, _I, _P, _I, _I],
    "trsm": [_I, _I, _I, _I, _I, _I, "scalar", _P, _I, _I, _P, _I, _I],
}

DRIVER_SIGNATURE = [_I, _I, _I, "scalar", _P, _I, _I, _P, _I, _I, "scalar", _P, _I, _I,
                    ctypes.POINTER(Product)]

EXTENSIONS = {
    "mublis_b200_init": ([], _I),
    "mublis_b200_last_error": ([], ctypes.c_char_p),
    "mublis_b200_set_stream": ([_P], _I),
    "mublis_b200_get_stream": ([], _P),
    "mublis_b200_set_form": ([ctypes.c_char, ctypes.c_char_p], _I),
    "mublis_b200_launch_count": ([], ctypes.c_ulonglong),
    "mublis_b200_profile_enable": ([_I], _I),
    "mublis_b200_profile_read": ([ctypes.c_char_p, ctypes.c_ulong], _I),
    "mublis_b200_test_stall_next": ([ctypes.c_ulonglong], _I),
    "mublis_b200_ozaki2_autotune": ([ctypes.c_char, _I, _I, _I, _I, _I, _P, _I, _I, _P, _I, _I,
                                     ctypes.c_double, ctypes.POINTER(_I),
                                     ctypes.POINTER(ctypes.c_double)], _I),
    "mublis_b200_fill_s": ([_P, _L, _L, _L, _U32, _U32, _I], _I),
    "mublis_b200_fill_d": ([_P, _L, _L, _L, _U32, _U32, _I], _I),
    "mublis_get_context": ([_P], _I),
    "mublis_b200_gemm_grouped": ([ctypes.c_char, ctypes.POINTER(GemmProblem), _I], _I),
    "mublis_b200_trsm_grouped": ([ctypes.c_char, ctypes.POINTER(TrsmProblem), _I], _I),
    "mublis_b200_plan_gemm_grouped": ([ctypes.c_char, ctypes.POINTER(GemmProblem), _I,
                                       ctypes.POINTER(_P)], _I),
    "mublis_b200_plan_trsm_grouped": ([ctypes.c_char, ctypes.POINTER(TrsmProblem), _I,
                                       ctypes.POINTER(_P)], _I),
    "mublis_b200_plan_run": ([_P], _I),
    "mublis_b200_plan_destroy": ([_P], _I),
    "mublis_b200_server_create": ([ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)], _I),
    "mublis_b200_server_destroy": ([_P], _I),
    "mublis_b200_server_attach": ([_P], _I),
    "mublis_b200_server_alloc": ([_P, ctypes.c_size_t, ctypes.POINTER(_P)], _I),
    "mublis_b200_server_free": ([_P, _P], _I),
    "mublis_b200_server_stats": ([_P, ctypes.POINTER(ServerStats)], _I),
    "mublis_b200_server_reset_stats": ([_P], _I),
    "mublis_b200_tune_save": ([ctypes.c_char_p], _I),
    "mublis_b200_tune_load": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)], _I),
    "mublis_b200_tune_reset": ([], _I),
    "mublis_b200_sgemm_noalloc": ([_I, _I, _I, _I, _I, ctypes.c_float, _P, _I, _I, _P, _I, _I,
                                   ctypes.c_float, _P, _I, _I], _I),
}

SCALARS = {"s": ctypes.c_float, "d": ctypes.c_double}


def declare(lib: ctypes.CDLL, optional_extensions: dict | None = None) -> ctypes.CDLL:
    """Declare argtypes/restype of every exported entry point on ``lib``."""
    for prefix, scalar in SCALARS.items():
        for routine, sig in CBLAS_SIGNATURES.items():
            fn = getattr(lib, f"cblas_{prefix}{routine}")
            fn.argtypes = [scalar if a == "scalar" else a for a in sig]
            fn.restype = None
        for routine, sig in MUBLIS_SIGNATURES.items():
            fn = getattr(lib, f"mublis_{prefix}{routine}")
            fn.argtypes = [scalar if a == "scalar" else a for a in sig]
            fn.restype = _I
        fn = getattr(lib, f"mublis_l3_{prefix}driver")
        fn.argtypes = [scalar if a == "scalar" else a for a in DRIVER_SIGNATURE]
        fn.restype = _I
    for name, (args, res) in {**EXTENSIONS, **(optional_extensions or {})}.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


_LIB = None


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load libmublis.so (built in-tree by ``make -C mublis_b200``).

    Raises FileNotFoundError if the library is missing: there is no CPU or
    Python fallback for any routine.
    """
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else Path(os.environ.get("MUBLIS_B200_LIB", LIB_PATH))
    if not p.is_file():
        raise FileNotFoundError(
            f"libmublis.so not found at {p}; build it with `make -C mublis_b200` "
            "(the B200 library has no fallback implementation)")
    lib = declare(ctypes.CDLL(str(p)))
    if path is None:
        _LIB = lib
    return lib


def last_error(lib: ctypes.CDLL | None = None) -> str:
    lib = lib or load()
    msg = lib.mublis_b200_last_error()
    return msg.decode() if msg else ""


def check(status: int, lib: ctypes.CDLL | None = None) -> None:
    if status != 0:
        raise RuntimeError(f"libmublis status {status}: {last_error(lib)}")
