"""Checker-side access to the oracle (test infrastructure only).

Two independent CPU implementations of the reference's Level-3 semantics:

* ``restated()`` -- ``oracle/lib/liboracle.so``, our C restatement
  (``oracle/mublis_oracle.c``), long-double accumulation, exported as
  ``oracle_{s,d}{gemm,symm,syrk,syr2k,trmm,trsm}`` / ``oracle_l3_{s,d}driver``
  with the reference's ``mublis_*`` argument lists;
* ``reference(config)`` -- the reference's own sources compiled by
  ``oracle/Makefile`` into ``oracle/_ref/<config>/libmublis.so`` (configs
  ``reference`` and ``avx2``), called through its ``cblas_*`` / ``mublis_*``.

Only tests, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline leg
use this module, and only as the thing the B200 library is checked against.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
RESTATED_LIB = HERE / "lib" / "liboracle.so"
REF_BENCH = HERE / "lib" / "ref_bench"


def ref_lib_path(config: str = "avx2") -> Path:
    return HERE / "_ref" / config / "libmublis.so"


_I, _P, _L, _D = ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_double
_SC = {"s": ctypes.c_float, "d": ctypes.c_double}

# Same argument lists as mublis.h (the restatement keeps them).
_MUBLIS = {
    "gemm": [_I, _I, _I, _I, _I, "s", _P, _I, _I, _P, _I, _I, "s", _P, _I, _I],
    "symm": [_I, _I, _I, _I, "s", _P, _I, _I, _P, _I, _I, "s", _P, _I, _I],
    "syrk": [_I, _I, _I, _I, "s", _P, _I, _I, "s", _P, _I, _I],
    "syr2k": [_I, _I, _I, _I, "s", _P, _I, _I, _P, _I, _I, "s", _P, _I, _I],
    "trmm": [_I, _I, _I, _I, _I, _I, "s", _P, _I, _I, _P, _I, _I],
    "trsm": [_I, _I, _I, _I, _I, _I, "s", _P, _I, _I, _P, _I, _I],
    "l3_driver": [_I, _I, _I, "s", _P, _I, _I, _P, _I, _I, "s", _P, _I, _I, _P],
}
_CBLAS = {
    "gemm": [_I, _I, _I, _I, _I, _I, "s", _P, _I, _P, _I, "s", _P, _I],
    "symm": [_I, _I, _I, _I, _I, "s", _P, _I, _P, _I, "s", _P, _I],
    "syrk": [_I, _I, _I, _I, _I, "s", _P, _I, "s", _P, _I],
    "syr2k": [_I, _I, _I, _I, _I, "s", _P, _I, _P, _I, "s", _P, _I],
    "trmm": [_I, _I, _I, _I, _I, _I, _I, "s", _P, _I, _P, _I],
    "trsm": [_I, _I, _I, _I, _I, _I, _I, "s", _P, _I, _P, _I],
}


def _sig(args, prefix):
    return [_SC[prefix] if a == "s" else a for a in args]


_restated = None


def restated() -> ctypes.CDLL:
    global _restated
    if _restated is None:
        if not RESTATED_LIB.is_file():
            raise FileNotFoundError(f"{RESTATED_LIB} missing: run `make -C oracle`")
        lib = ctypes.CDLL(str(RESTATED_LIB))
        for p in "sd":
            for r, args in _MUBLIS.items():
                name = f"oracle_l3_{p}driver" if r == "l3_driver" else f"oracle_{p}{r}"
                fn = getattr(lib, name)
                fn.argtypes = _sig(args, p)
                fn.restype = _I
        lib.oracle_set_threads.argtypes = [_I]
        lib.oracle_fill_s.argtypes = [_P, _L, _L, _L, ctypes.c_uint32, ctypes.c_uint32, _I]
        lib.oracle_fill_d.argtypes = [_P, _L, _L, _L, ctypes.c_uint32, ctypes.c_uint32, _I]
        lib.oracle_philox.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, _P]
        lib.oracle_philox_ctr.argtypes = [_P, _P, _P]
        lib.oracle_dd_gemm_entries.argtypes = [_I, _I, _I, _L, _D, _P, _L, _P, _L, _D, _P, _L,
                                               _L, _P, _P, _P, _P]
        _restated = lib
    return _restated


_refs: dict = {}


def reference(config: str = "avx2") -> ctypes.CDLL:
    """The reference's own build (CPU) as a ctypes library."""
    if config not in _refs:
        path = ref_lib_path(config)
        if not path.is_file():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the "
                                    "reference sources are present")
        lib = ctypes.CDLL(str(path))
        for p in "sd":
            for r, args in _CBLAS.items():
                fn = getattr(lib, f"cblas_{p}{r}")
                fn.argtypes = _sig(args, p)
                fn.restype = None
            for r, args in _MUBLIS.items():
                name = f"mublis_l3_{p}driver" if r == "l3_driver" else f"mublis_{p}{r}"
                fn = getattr(lib, name)
                fn.argtypes = _sig(args, p)
                fn.restype = _I
        _refs[config] = lib
    return _refs[config]


def set_threads(n: int) -> None:
    restated().oracle_set_threads(int(n))


# ---- seeded inputs ---------------------------------------------------------

UNIFORM, WIDE, DIAG = 0, 1, 2


def philox(index: int, seed: int, matrix_id: int) -> tuple:
    out = (ctypes.c_uint32 * 4)()
    restated().oracle_philox(index, seed, matrix_id, out)
    return tuple(out)


def philox_ctr(ctr, key) -> tuple:
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    out = (ctypes.c_uint32 * 4)()
    restated().oracle_philox_ctr(c, k, out)
    return tuple(out)


def fill(m: int, n: int, dtype, seed: int, matrix_id: int, kind: int = UNIFORM) -> np.ndarray:
    """m x n column-major (Fortran-order) seeded matrix."""
    dt = np.dtype(dtype)
    x = np.empty((m, n), dtype=dt, order="F")
    fn = restated().oracle_fill_s if dt == np.float32 else restated().oracle_fill_d
    if m and n:
        fn(x.ctypes.data, m, n, m, seed, matrix_id, kind)
    return x


def trsm_matrix(n: int, dtype, seed: int, matrix_id: int) -> np.ndarray:
    """Well-conditioned triangular-solve operand: off-diagonals uniform[-1,1)/n,
    diagonal uniform[1,2) (same Philox stream, element-wise)."""
    a = fill(n, n, dtype, seed, matrix_id, UNIFORM) / np.asarray(n, dtype=dtype)
    d = fill(n, n, dtype, seed, matrix_id, DIAG)
    idx = np.arange(n)
    a[idx, idx] = d[idx, idx]
    return np.asfortranarray(a.astype(dtype))


def dd_gemm_entries(a, b, rows, cols, alpha=1.0, beta=0.0, c0=None, ta=False, tb=False,
                    threads=None):
    """Double-double values of selected entries of alpha*op(A)op(B)+beta*C0
    (A, B, C0 column-major float32/float64); returns (hi, lo) arrays.  The
    entries are split over `threads` host threads (default: all cores); the
    C routine runs without the GIL."""
    a = np.asfortranarray(a)
    b = np.asfortranarray(b)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    hi = np.empty(len(rows))
    lo = np.empty(len(rows))
    k = a.shape[0] if ta else a.shape[1]
    is32 = 1 if a.dtype == np.float32 else 0
    cptr, ldc = (None, 1)
    if c0 is not None and beta != 0:
        c0 = np.asfortranarray(c0)
        cptr, ldc = c0.ctypes.data, c0.shape[0]
    fn = restated().oracle_dd_gemm_entries
    count = len(rows)
    nt = max(1, min(threads or os.cpu_count() or 1, count // 64 or 1))
    bounds = [count * t // nt for t in range(nt + 1)]

    def part(t):
        q0, q1 = bounds[t], bounds[t + 1]
        if q1 > q0:
            fn(is32, int(ta), int(tb), k, alpha, a.ctypes.data, a.shape[0], b.ctypes.data,
               b.shape[0], beta, cptr, ldc, q1 - q0, rows.ctypes.data + 8 * q0,
               cols.ctypes.data + 8 * q0, hi.ctypes.data + 8 * q0, lo.ctypes.data + 8 * q0)

    if nt == 1:
        part(0)
    else:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(nt) as ex:
            list(ex.map(part, range(nt)))
    return hi, lo
