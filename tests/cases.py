"""Shared Level-3 test cases (inputs, calls, error metrics).

A *case* is a plain dict:
    routine  gemm | symm | syrk | syr2k | trmm | trsm
    dtype    "float32" | "float64"
    order    "F" (column-major) | "C" (row-major)
    m, n, k  sizes (k used by gemm/syrk/syr2k)
    ta, tb   transposes (gemm: both; syrk/syr2k/trmm/trsm: ta)
    right, lower, unit   side / uplo / diag flags
    alpha, beta
    seed     Philox seed (inputs from oracle.fill, matrix ids 0, 1, 2)
    draw     "uniform" (default) or "normal" (numpy default_rng(seed), as the
             reference's check_cblas.py:155-163 does)

Input construction follows the reference's tests (check_cblas.py:192-222):
the unstored triangle of a symmetric operand is NaN, the unused triangle of a
triangular operand is NaN, and a unit diagonal is NaN, so any read of them
shows up in the result.
"""
from __future__ import annotations

import ctypes
import itertools

import numpy as np

import mublis_b200 as mb
from oracle import oracle as orc

EPS = {np.dtype(np.float32): 2.0 ** -24, np.dtype(np.float64): 2.0 ** -53}
# The reference test-suite tolerances (check_cblas.py:24-37).
REF_TOL = {np.dtype(np.float32): (5e-4, 5e-5), np.dtype(np.float64): (2e-11, 1e-12)}


def _draw(case, shape, matrix_id):
    dt = np.dtype(case["dtype"])
    if case.get("draw") == "normal":
        rng = np.random.default_rng(case["seed"] * 7 + matrix_id)
        return rng.standard_normal(shape).astype(dt)
    return orc.fill(shape[0], shape[1], dt, case["seed"], matrix_id)


def shapes(case):
    r, m, n, k = case["routine"], case["m"], case["n"], case["k"]
    if r == "gemm":
        a = (k, m) if case["ta"] else (m, k)
        b = (n, k) if case["tb"] else (k, n)
        return a, b, (m, n)
    if r == "symm":
        s = n if case["right"] else m
        return (s, s), (m, n), (m, n)
    if r in ("syrk", "syr2k"):
        a = (k, n) if case["ta"] else (n, k)
        return a, a, (n, n)
    s = n if case["right"] else m
    return (s, s), None, (m, n)  # trmm/trsm: B is the in/out operand


def build(case):
    """Inputs (a, b, c0) as arrays in case['order']; b is None for trmm/trsm
    (c0 is their B)."""
    dt = np.dtype(case["dtype"])
    sa, sb, sc = shapes(case)
    r = case["routine"]
    a = _draw(case, sa, 0).astype(np.float64)
    if r == "symm":
        tri = np.triu_indices(sa[0], 1) if case["lower"] else np.tril_indices(sa[0], -1)
        a[tri] = np.nan
    if r in ("trmm", "trsm"):
        s = sa[0]
        if r == "trsm" and case.get("draw") != "normal":
            a = orc.trsm_matrix(s, np.float64, case["seed"], 0)
        elif case.get("draw") == "normal":
            rng = np.random.default_rng(case["seed"])
            a = rng.uniform(-0.25, 0.25, size=(s, s))
            np.fill_diagonal(a, rng.uniform(1.5, 2.5, size=s))
        tri = np.triu_indices(s, 1) if case["lower"] else np.tril_indices(s, -1)
        a[tri] = np.nan
        if case["unit"]:
            np.fill_diagonal(a, np.nan)
    b = None if sb is None else _draw(case, sb, 1)
    c0 = _draw(case, sc, 2)
    o = case["order"]
    a = np.array(a, dtype=dt, order=o)
    b = None if b is None else np.array(b, dtype=dt, order=o)
    c0 = np.array(c0, dtype=dt, order=o)
    return a, b, c0


def ld(x, order):
    """Leading dimension as the reference test computes it
    (check_cblas.py:171-173)."""
    if x is None:
        return 1
    axis = 0 if order == "C" else 1
    if x.size == 0 or x.shape[axis] == 1:
        # a single row/column: the stride along it is meaningless
        return max(1, x.shape[1 - axis])
    return max(1, x.strides[axis] // x.itemsize)


def _ptr(x):
    return ctypes.c_void_p(x.ctypes.data) if x is not None else None


def cblas_call(lib, case, a, b, c):
    """Run the case through a library's cblas_* (our libmublis or the
    reference build); c is updated in place."""
    dt = np.dtype(case["dtype"])
    p = "s" if dt == np.float32 else "d"
    order = mb.ROW if case["order"] == "C" else mb.COL
    r = case["routine"]
    T = lambda f: mb.TRANS if f else mb.NO_TRANS
    U = mb.LOWER if case.get("lower") else mb.UPPER
    S = mb.RIGHT if case.get("right") else mb.LEFT
    D = mb.UNIT if case.get("unit") else mb.NON_UNIT
    al, be = case["alpha"], case.get("beta", 0.0)
    o = case["order"]
    fn = getattr(lib, f"cblas_{p}{r}")
    if r == "gemm":
        fn(order, T(case["ta"]), T(case["tb"]), case["m"], case["n"], case["k"], al, _ptr(a),
           ld(a, o), _ptr(b), ld(b, o), be, _ptr(c), ld(c, o))
    elif r == "symm":
        fn(order, S, U, case["m"], case["n"], al, _ptr(a), ld(a, o), _ptr(b), ld(b, o), be, _ptr(c),
           ld(c, o))
    elif r == "syrk":
        fn(order, U, T(case["ta"]), case["n"], case["k"], al, _ptr(a), ld(a, o), be, _ptr(c), ld(c, o))
    elif r == "syr2k":
        fn(order, U, T(case["ta"]), case["n"], case["k"], al, _ptr(a), ld(a, o), _ptr(b), ld(b, o), be,
           _ptr(c), ld(c, o))
    else:
        fn(order, S, U, T(case["ta"]), D, case["m"], case["n"], al, _ptr(a), ld(a, o), _ptr(c),
           ld(c, o))


def _strides(x):
    return x.strides[0] // x.itemsize, x.strides[1] // x.itemsize


def oracle_call(case, a, b, c):
    """Run the case through the oracle restatement (mublis-level functions
    with the arrays' own element strides, so row-major needs no remapping)."""
    lib = orc.restated()
    dt = np.dtype(case["dtype"])
    p = "s" if dt == np.float32 else "d"
    r = case["routine"]
    tr = lambda f: mb.M_TRANSPOSE if f else mb.M_NO_TRANSPOSE
    up = mb.M_LOWER if case.get("lower") else mb.M_UPPER
    sd = mb.M_RIGHT if case.get("right") else mb.M_LEFT
    dg = mb.M_UNIT if case.get("unit") else mb.M_NON_UNIT
    al, be = case["alpha"], case.get("beta", 0.0)
    fn = getattr(lib, f"oracle_{p}{r}")
    ra, ca = _strides(a)
    rc, cc = _strides(c)
    if b is not None:
        rb, cb = _strides(b)
    if r == "gemm":
        st = fn(tr(case["ta"]), tr(case["tb"]), case["m"], case["n"], case["k"], al, _ptr(a), ra,
                ca, _ptr(b), rb, cb, be, _ptr(c), rc, cc)
    elif r == "symm":
        st = fn(sd, up, case["m"], case["n"], al, _ptr(a), ra, ca, _ptr(b), rb, cb, be, _ptr(c),
                rc, cc)
    elif r == "syrk":
        st = fn(up, tr(case["ta"]), case["n"], case["k"], al, _ptr(a), ra, ca, be, _ptr(c), rc, cc)
    elif r == "syr2k":
        st = fn(up, tr(case["ta"]), case["n"], case["k"], al, _ptr(a), ra, ca, _ptr(b), rb, cb, be,
                _ptr(c), rc, cc)
    else:
        st = fn(sd, up, tr(case["ta"]), dg, case["m"], case["n"], al, _ptr(a), ra, ca, _ptr(c),
                rc, cc)
    assert st == 0


def scipy_expected(case, a, b, c0):
    """The reference test-suite's own oracle: scipy.linalg.blas
    (check_cblas.py:179-180)."""
    from scipy.linalg import blas
    dt = np.dtype(case["dtype"])
    r = case["routine"]
    f = lambda x: np.array(x, dtype=dt, order="F", copy=True)
    fn = blas.get_blas_funcs(r, dtype=dt)
    al, be = case["alpha"], case.get("beta", 0.0)
    if r == "gemm":
        return fn(al, f(a), f(b), beta=be, c=f(c0), trans_a=int(case["ta"]),
                  trans_b=int(case["tb"]), overwrite_c=1)
    if r == "symm":
        return fn(al, f(a), f(b), beta=be, c=f(c0), side=int(case["right"]),
                  lower=int(case["lower"]), overwrite_c=1)
    if r == "syrk":
        return fn(al, f(a), beta=be, c=f(c0), trans=int(case["ta"]), lower=int(case["lower"]),
                  overwrite_c=1)
    if r == "syr2k":
        return fn(al, f(a), f(b), beta=be, c=f(c0), trans=int(case["ta"]),
                  lower=int(case["lower"]), overwrite_c=1)
    return fn(al, f(a), f(c0), side=int(case["right"]), lower=int(case["lower"]),
              trans_a=int(case["ta"]), diag=int(case["unit"]), overwrite_b=1)


def active_mask(case):
    """Elements the routine writes (SYRK/SYR2K: the uplo triangle)."""
    sc = shapes(case)[2]
    mask = np.ones(sc, dtype=bool)
    if case["routine"] in ("syrk", "syr2k"):
        mask = np.tril(mask) if case["lower"] else np.triu(mask)
    return mask


def inner_dim(case):
    r = case["routine"]
    if r in ("gemm", "syrk", "syr2k"):
        return case["k"] * (2 if r == "syr2k" else 1)
    if r == "symm":
        return case["n"] if case["right"] else case["m"]
    return case["n"] if case["right"] else case["m"]


def normwise_error(case, actual, expected, a, b, c0):
    """||C - C_ref||_F / (|alpha| ||A||_F ||B||_F + |beta| ||C0||_F) over the
    written part; for TRSM the relative forward error ||X - X_ref|| / ||X_ref||."""
    mask = active_mask(case)
    diff = np.where(mask, np.asarray(actual, np.float64) - np.asarray(expected, np.float64), 0)
    num = np.linalg.norm(diff)
    if case["routine"] == "trsm":
        den = np.linalg.norm(np.where(mask, np.asarray(expected, np.float64), 0))
        return num / max(den, 1e-300)
    fa = np.linalg.norm(np.nan_to_num(np.asarray(a, np.float64)))
    if case["routine"] in ("trmm",):
        fb = np.linalg.norm(np.asarray(c0, np.float64))
        den = abs(case["alpha"]) * fa * fb
    else:
        fb = np.linalg.norm(np.asarray(b if b is not None else a, np.float64))
        if case["routine"] == "syr2k":
            fb *= 2 ** 0.5
        den = abs(case["alpha"]) * fa * fb + abs(case.get("beta", 0.0)) * np.linalg.norm(
            np.asarray(c0, np.float64))
    return num / max(den, 1e-300)


def reference_matrix(small_m=5, small_n=4, small_k=3):
    """The reference test-suite's case matrix (check_cblas.py:224-473): every
    routine, both precisions, both layouts and every flag combination."""
    out = []
    for dt, order in itertools.product(("float32", "float64"), ("C", "F")):
        base = dict(dtype=dt, order=order, seed=314159, draw="normal")
        for ta, tb in itertools.product((False, True), repeat=2):
            out.append(dict(base, routine="gemm", m=small_m, n=small_n, k=small_k, ta=ta, tb=tb,
                            alpha=1.25, beta=-0.5))
        for right, lower in itertools.product((False, True), repeat=2):
            out.append(dict(base, routine="symm", m=5, n=3, k=0, right=right, lower=lower,
                            alpha=0.75, beta=-0.25))
        for ta, lower in itertools.product((False, True), repeat=2):
            out.append(dict(base, routine="syrk", m=5, n=5, k=3, ta=ta, lower=lower, alpha=1.25,
                            beta=-0.5))
            out.append(dict(base, routine="syr2k", m=5, n=5, k=3, ta=ta, lower=lower,
                            alpha=0.75, beta=-0.25))
        for r in ("trmm", "trsm"):
            for right, lower, ta, unit in itertools.product((False, True), repeat=4):
                out.append(dict(base, routine=r, m=5, n=3, k=0, right=right, lower=lower, ta=ta,
                                unit=unit, alpha=0.75))
    return out


def case_id(c):
    flags = "".join(f for f, on in (("T", c.get("ta")), ("t", c.get("tb")), ("R", c.get("right")),
                                    ("L", c.get("lower")), ("U", c.get("unit"))) if on)
    return f"{c['routine']}-{c['dtype'][5:]}-{c['order']}-{c['m']}x{c['n']}x{c['k']}-{flags or '_'}"
