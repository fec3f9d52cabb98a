"""Parity of the B200 library with the oracle, through the C ABI (GPU).

Tolerances (stated per test):
  * the reference test-suite's own case matrix: its assert_allclose
    tolerances (f32 rtol 5e-4 / atol 5e-5, f64 rtol 2e-11 / atol 1e-12);
  * everything else: normwise relative error <= 4 * k * u (u = 2^-24 for
    FP32, 2^-53 for FP64; k the inner dimension, the order for TRSM, where
    the bound is on the relative forward error of these well-conditioned
    systems) against the long-double oracle restatement or the golden
    outputs of the reference build;
  * untouched parts (the opposite triangle of SYRK/SYR2K) bit-identical.
"""
import ctypes
import itertools
import json
import threading
from pathlib import Path

import numpy as np
import pytest

import mublis_b200 as mb
from oracle import oracle as orc
from tests import cases as cs

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "l3_golden.npz"
REF_MATRIX = cs.reference_matrix()


@pytest.fixture(scope="module", autouse=True)
def plain_forms(lib):
    assert lib.mublis_b200_init() == 0, mb.last_error(lib)
    lib.mublis_b200_set_form(b"s", b"plain")
    lib.mublis_b200_set_form(b"d", b"plain")
    orc.set_threads(8)
    yield


def run_lib(lib, case):
    a, b, c0 = cs.build(case)
    out = c0.copy(order="K")
    cs.cblas_call(lib, case, a, b, out)
    return a, b, c0, out


def run_oracle(case):
    a, b, c0 = cs.build(case)
    out = c0.copy(order="K")
    cs.oracle_call(case, a, b, out)
    return out


def tol_of(case):
    return 4 * max(cs.inner_dim(case), 1) * cs.EPS[np.dtype(case["dtype"])]


@pytest.mark.parametrize("case", REF_MATRIX, ids=[cs.case_id(c) for c in REF_MATRIX])
def test_reference_suite_matrix(lib, case):
    """check_cblas.py's 192 cases, same inputs style (NaN-poisoned unused
    triangles and unit diagonals), same oracle (scipy) and tolerances."""
    a, b, c0, out = run_lib(lib, case)
    expected = np.asarray(cs.scipy_expected(case, a, b, c0))
    rtol, atol = cs.REF_TOL[np.dtype(case["dtype"])]
    mask = cs.active_mask(case)
    np.testing.assert_allclose(out[mask], expected[mask], rtol=rtol, atol=atol)
    np.testing.assert_array_equal(out[~mask], c0[~mask])


def _golden():
    data = np.load(GOLDEN)
    return json.loads(str(data["cases"])), data


GOLDEN_CASES, _ = _golden()


@pytest.mark.parametrize("idx", range(len(GOLDEN_CASES)),
                         ids=[cs.case_id(c) for c in GOLDEN_CASES])
def test_golden(lib, idx):
    """Outputs of the reference's avx2 build on seeded inputs."""
    cases, data = _golden()
    case = cases[idx]
    expected = data[f"out{idx}"]
    a, b, c0, out = run_lib(lib, case)
    if out.size == 0:
        return
    mask = cs.active_mask(case)
    err = cs.normwise_error(case, out, expected, a, b, c0)
    assert err <= tol_of(case), (err, tol_of(case))
    np.testing.assert_array_equal(out[~mask], expected[~mask])
    assert np.isfinite(out[mask]).all()


RAGGED = [1, 7, 127, 129, 255]


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("ta,tb", list(itertools.product((False, True), repeat=2)))
@pytest.mark.parametrize("mnk", [(127, 129, 255), (255, 7, 129), (1, 255, 127), (129, 1, 1),
                                 (300, 200, 513)])
def test_gemm_ragged(lib, dtype, ta, tb, mnk):
    m, n, k = mnk
    case = dict(routine="gemm", dtype=dtype, order="F", m=m, n=n, k=k, ta=ta, tb=tb,
                alpha=0.75, beta=0.25, seed=5)
    a, b, c0, out = run_lib(lib, case)
    ref = run_oracle(case)
    assert cs.normwise_error(case, out, ref, a, b, c0) <= tol_of(case)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("routine,flags", [
    ("symm", dict(right=False, lower=True)), ("symm", dict(right=True, lower=False)),
    ("syrk", dict(ta=False, lower=True)), ("syrk", dict(ta=True, lower=False)),
    ("syr2k", dict(ta=False, lower=True)), ("syr2k", dict(ta=True, lower=False)),
    ("trmm", dict(right=False, lower=True, ta=False, unit=False)),
    ("trmm", dict(right=True, lower=False, ta=True, unit=True)),
    ("trsm", dict(right=False, lower=True, ta=False, unit=False)),
    ("trsm", dict(right=False, lower=False, ta=True, unit=False)),
    ("trsm", dict(right=True, lower=True, ta=True, unit=True)),
    ("trsm", dict(right=True, lower=False, ta=False, unit=False)),
])
@pytest.mark.parametrize("order", ["F", "C"])
def test_family_midsize(lib, dtype, routine, flags, order):
    """Sizes that cross tile and leaf boundaries (and the TRSM recursion)."""
    case = dict(routine=routine, dtype=dtype, order=order, m=301, n=177, k=211, alpha=0.75,
                beta=0.25, seed=8, **flags)
    if routine in ("syrk", "syr2k"):
        case["m"] = case["n"]
    if routine == "trmm" and flags.get("unit"):
        pass
    a, b, c0, out = run_lib(lib, case)
    ref = run_oracle(case)
    mask = cs.active_mask(case)
    assert np.isfinite(out[mask]).all()
    assert cs.normwise_error(case, out, ref, a, b, c0) <= tol_of(case)
    np.testing.assert_array_equal(out[~mask], c0[~mask])


@pytest.mark.parametrize("p", ["s", "d"])
def test_beta_zero_never_reads_c(lib, p):
    dt = np.float32 if p == "s" else np.float64
    a = orc.fill(65, 33, dt, 1, 0)
    b = orc.fill(33, 70, dt, 1, 1)
    c = np.full((65, 70), np.nan, dtype=dt, order="F")
    st = getattr(lib, f"mublis_{p}gemm")(0, 0, 65, 70, 33, 1.5, a.ctypes.data, 1, 65,
                                         b.ctypes.data, 1, 33, 0.0, c.ctypes.data, 1, 65)
    assert st == 0
    assert np.isfinite(c).all()
    ref = 1.5 * (a.astype(np.float64) @ b.astype(np.float64))
    err = np.linalg.norm(c - ref) / (1.5 * np.linalg.norm(a) * np.linalg.norm(b))
    assert err <= 4 * 33 * cs.EPS[np.dtype(dt)]


@pytest.mark.parametrize("p", ["s", "d"])
def test_alpha_zero_never_reads_ab(lib, p):
    dt = np.float32 if p == "s" else np.float64
    a = np.full((40, 30), np.nan, dtype=dt, order="F")
    b = np.full((30, 20), np.nan, dtype=dt, order="F")
    c0 = orc.fill(40, 20, dt, 2, 2)
    c = c0.copy(order="F")
    st = getattr(lib, f"mublis_{p}gemm")(0, 0, 40, 20, 30, 0.0, a.ctypes.data, 1, 40,
                                         b.ctypes.data, 1, 30, 0.5, c.ctypes.data, 1, 40)
    assert st == 0
    np.testing.assert_array_equal(c, (c0 * dt(0.5)).astype(dt))


@pytest.mark.parametrize("p", ["s", "d"])
def test_empty_sizes_are_noops(lib, p):
    dt = np.float32 if p == "s" else np.float64
    c = orc.fill(5, 5, dt, 3, 2)
    keep = c.copy()
    fn = getattr(lib, f"mublis_{p}gemm")
    assert fn(0, 0, 0, 5, 3, 1.0, None, 1, 1, None, 1, 1, 0.0, c.ctypes.data, 1, 5) == 0
    assert fn(0, 0, 5, 0, 3, 1.0, None, 1, 1, None, 1, 1, 0.0, c.ctypes.data, 1, 5) == 0
    np.testing.assert_array_equal(c, keep)
    # k == 0: C := beta * C
    assert fn(0, 0, 5, 5, 0, 1.0, None, 1, 1, None, 1, 1, 0.5, c.ctypes.data, 1, 5) == 0
    np.testing.assert_array_equal(c, keep * dt(0.5))


@pytest.mark.parametrize("p", ["s", "d"])
def test_general_strides(lib, p):
    """mublis_* accept any (rs, cs): strided views in both orientations and
    padded non-unit strides on both axes."""
    dt = np.float32 if p == "s" else np.float64
    m, n, k = 45, 38, 29
    big_a = orc.fill(3 * m, 2 * k + 1, dt, 4, 0)
    big_b = orc.fill(k, 5 * n, dt, 4, 1)
    big_c = orc.fill(2 * m, 3 * n, dt, 4, 2)
    a = big_a[::3, 1::2]                         # rs = 3, cs = 6m (gathered)
    b = big_b[:, ::5]                            # rs = 1, cs = 5k
    c0 = np.ascontiguousarray(big_c[::2, ::3])   # row-major: rs = n, cs = 1
    c = c0.copy()
    el = np.dtype(dt).itemsize
    (ars, acs), (brs, bcs), (crs, ccs) = [(x.strides[0] // el, x.strides[1] // el)
                                          for x in (a, b, c)]
    st = getattr(lib, f"mublis_{p}gemm")(0, 0, m, n, k, 0.75, a.ctypes.data, ars, acs,
                                         b.ctypes.data, brs, bcs, 0.25, c.ctypes.data, crs, ccs)
    assert st == 0
    ref = 0.75 * (a.astype(np.float64) @ b.astype(np.float64)) + 0.25 * c0
    err = np.linalg.norm(c - ref) / (0.75 * np.linalg.norm(a) * np.linalg.norm(b) +
                                     0.25 * np.linalg.norm(c0))
    assert err <= 4 * k * cs.EPS[np.dtype(dt)]


# The generic driver's whole case matrix: every (jp, ji, pi) relation triple
# (ALL / LOWER / UPPER each) with every operand structure (GENERAL,
# SYMMETRIC, TRIANGULAR) for A and for B.  The stored triangle of a
# structured operand and a triangular operand's unit diagonal alternate with
# the case index, so both triangles and both diagonal treatments occur.
def _driver_matrix():
    out = []
    for idx, (jp, ji, pi, sa, sb) in enumerate(itertools.product(range(3), range(3), range(3),
                                                                 range(3), range(3))):
        def operand(struc, salt):
            if struc == 0:
                return (0, 0, 0)
            uplo = 1 + (idx + salt) % 2
            diag = (idx // 2 + salt) % 2 if struc == 2 else 0
            return (struc, uplo, diag)
        out.append(dict(jp=jp, ji=ji, pi=pi, a=operand(sa, 0), b=operand(sb, 1)))
    return out


DRIVER_MATRIX = _driver_matrix()


def _driver_id(dc):
    names = "AlU"
    s = "GST"
    return (f"jp{names[dc['jp']]}-ji{names[dc['ji']]}-pi{names[dc['pi']]}-"
            f"a{s[dc['a'][0]]}{dc['a'][1]}{dc['a'][2]}-b{s[dc['b'][0]]}{dc['b'][1]}{dc['b'][2]}")


@pytest.mark.parametrize("p", ["s", "d"])
@pytest.mark.parametrize("dc", DRIVER_MATRIX, ids=[_driver_id(d) for d in DRIVER_MATRIX])
def test_generic_driver_domains(lib, p, dc):
    """mublis_l3_{s,d}driver on the device against the oracle's driver
    (element-wise domain semantics of l3_driver.c:49-256 and packm.c:40-71)
    for every domain relation triple and operand structure; the unstored
    triangles and unit diagonals are NaN.  Normwise error <= 4 k u and the
    part of C outside ji bit-identical to its input."""
    dt = np.float32 if p == "s" else np.float64
    m = n = k = 161
    a = orc.fill(m, k, dt, 3, 0)
    b = orc.fill(k, n, dt, 3, 1)
    c0 = orc.fill(m, n, dt, 3, 2)
    for x, (struc, uplo, diag) in ((a, dc["a"]), (b, dc["b"])):
        if struc in (1, 2):
            tri = np.triu_indices(k, 1) if uplo == 1 else np.tril_indices(k, -1)
            x[tri] = np.nan
        if struc == 2 and diag == 1:
            np.fill_diagonal(x, np.nan)
    prod = mb.Product(mb.Domain(dc["jp"], dc["ji"], dc["pi"]), mb.Operand(*dc["a"]),
                      mb.Operand(*dc["b"]))
    outs = []
    for fn in (getattr(orc.restated(), f"oracle_l3_{p}driver"), getattr(lib, f"mublis_l3_{p}driver")):
        c = c0.copy(order="F")
        assert fn(m, n, k, 0.75, a.ctypes.data, 1, m, b.ctypes.data, 1, k, 0.25, c.ctypes.data,
                  1, m, ctypes.byref(prod)) == 0
        outs.append(c)
    fa = np.linalg.norm(np.nan_to_num(a)) * np.linalg.norm(np.nan_to_num(b)) * 0.75
    err = np.linalg.norm(outs[0] - outs[1]) / (fa + 0.25 * np.linalg.norm(c0))
    assert np.isfinite(outs[1]).all()
    assert err <= 4 * k * cs.EPS[np.dtype(dt)]
    i, j = np.indices((m, n))
    outside = (j > i) if dc["ji"] == 1 else (j < i) if dc["ji"] == 2 else np.zeros((m, n), bool)
    np.testing.assert_array_equal(outs[1][outside], c0[outside])


def test_device_pointers_in_place(lib):
    """Device-resident operands are used in place (no staging)."""
    torch = pytest.importorskip("torch")
    m, n, k = 300, 257, 190
    a = orc.fill(m, k, np.float32, 6, 0)
    b = orc.fill(k, n, np.float32, 6, 1)
    c0 = orc.fill(m, n, np.float32, 6, 2)
    ta = torch.from_numpy(a.T.copy()).cuda()   # (k, m) row-major == a column-major
    tb = torch.from_numpy(b.T.copy()).cuda()
    tc = torch.from_numpy(c0.T.copy()).cuda()
    torch.cuda.synchronize()
    st = lib.mublis_sgemm(0, 0, m, n, k, 0.75, ta.data_ptr(), 1, m, tb.data_ptr(), 1, k, 0.25,
                          tc.data_ptr(), 1, m)
    assert st == 0
    out = tc.cpu().numpy().T
    case = dict(routine="gemm", dtype="float32", order="F", m=m, n=n, k=k, ta=False, tb=False,
                alpha=0.75, beta=0.25, seed=6)
    ref = run_oracle(case)
    assert cs.normwise_error(case, out, ref, a, b, c0) <= tol_of(case)


def test_sgemm_1024_seeded_case(lib):
    """Plain SGEMM NN, column-major, m=n=k=1024, alpha 1, beta 0.5, seed 0:
    normwise error <= 4 * 1024 * 2^-24 against the oracle."""
    case = dict(routine="gemm", dtype="float32", order="F", m=1024, n=1024, k=1024, ta=False,
                tb=False, alpha=1.0, beta=0.5, seed=0)
    a, b, c0, out = run_lib(lib, case)
    ref = run_oracle(case)
    err = cs.normwise_error(case, out, ref, a, b, c0)
    assert err <= 4 * 1024 * 2.0 ** -24, err


def test_concurrent_callers_match_serial(lib):
    """The library is thread-safe like the reference (pool.c:4-10): results
    from 8 concurrent host threads equal the single-threaded results."""
    cases = [dict(routine="gemm", dtype=dt, order="F", m=200 + 7 * i, n=150 + 3 * i,
                  k=100 + 11 * i, ta=bool(i % 2), tb=bool(i % 3 == 0), alpha=0.75, beta=0.25,
                  seed=40 + i) for i, dt in zip(range(8), itertools.cycle(["float32", "float64"]))]
    serial = [run_lib(lib, c)[3] for c in cases]
    results = [None] * len(cases)

    def work(i):
        results[i] = run_lib(lib, cases[i])[3]

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(cases))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for s, r in zip(serial, results):
        np.testing.assert_array_equal(s, r)


@pytest.mark.parametrize("p", ["s", "d"])
def test_context_micro_kernels(lib, p):
    """b200_context's device micro-kernels honour the packed-panel ABI of
    mublis_instantiate.h (gemm_ukr, gemmtrsm{l,u}_ukr)."""
    dt = np.float32 if p == "s" else np.float64
    ct = ctypes.c_float if p == "s" else ctypes.c_double

    class Ctx(ctypes.Structure):
        _fields_ = [("gemm", ctypes.c_void_p), ("trsml", ctypes.c_void_p),
                    ("trsmu", ctypes.c_void_p), ("mr", ctypes.c_int), ("nr", ctypes.c_int),
                    ("mc", ctypes.c_int), ("kc", ctypes.c_int), ("nc", ctypes.c_int)]

    class Both(ctypes.Structure):
        _fields_ = [("s", Ctx), ("d", Ctx)]

    both = Both()
    assert lib.mublis_get_context(ctypes.byref(both)) == 0
    ctx = both.s if p == "s" else both.d
    mr, nr, k = ctx.mr, ctx.nr, 13
    assert ctx.mc % mr == 0 and ctx.nc % nr == 0 and ctx.kc % mr == 0 and ctx.kc % nr == 0
    PT = ctypes.POINTER(ct)
    gemm_t = ctypes.CFUNCTYPE(None, ctypes.c_int, ct, PT, PT, ct, PT, ctypes.c_int, ctypes.c_int,
                              ctypes.c_void_p)
    apk = orc.fill(mr * k, 1, dt, 9, 0).ravel()
    bpk = orc.fill(nr * k, 1, dt, 9, 1).ravel()
    c0 = orc.fill(mr, nr, dt, 9, 2)
    c = c0.copy(order="F")
    gemm_t(ctx.gemm)(k, 0.5, apk.ctypes.data_as(PT), bpk.ctypes.data_as(PT), 2.0,
                     c.ctypes.data_as(PT), 1, mr, None)
    A = apk.reshape(k, mr).T.astype(np.float64)
    B = bpk.reshape(k, nr).astype(np.float64)
    np.testing.assert_allclose(c, 0.5 * A @ B + 2.0 * c0, rtol=1e-4 if p == "s" else 1e-12,
                               atol=1e-5 if p == "s" else 1e-13)

    trsm_t = ctypes.CFUNCTYPE(None, ctypes.c_int, ct, PT, PT, PT, PT, PT, ctypes.c_int,
                              ctypes.c_int, ctypes.c_void_p)
    for lower, fn in ((True, ctx.trsml), (False, ctx.trsmu)):
        a11 = np.tril(orc.fill(mr, mr, dt, 10, 3) / mr) if lower else np.triu(
            orc.fill(mr, mr, dt, 10, 3) / mr)
        diag = 1.0 + np.arange(mr, dtype=dt) / mr
        a11[np.arange(mr), np.arange(mr)] = (1.0 / diag).astype(dt)   # pre-inverted
        a11f = np.asfortranarray(a11.astype(dt))
        b11 = orc.fill(mr, nr, dt, 10, 4)                              # row-major packed
        b11p = np.ascontiguousarray(b11)
        c11 = np.zeros((mr, nr), dtype=dt, order="F")
        trsm_t(fn)(k, 0.75, apk.ctypes.data_as(PT), a11f.ctypes.data_as(PT),
                   bpk.ctypes.data_as(PT), b11p.ctypes.data_as(PT), c11.ctypes.data_as(PT), 1,
                   mr, None)
        R = 0.75 * b11.astype(np.float64) - A @ B
        L = a11.astype(np.float64).copy()
        L[np.arange(mr), np.arange(mr)] = diag
        X = np.linalg.solve(L, R)
        np.testing.assert_allclose(c11, X, rtol=1e-3 if p == "s" else 1e-11,
                                   atol=1e-4 if p == "s" else 1e-12)
        np.testing.assert_array_equal(b11p, c11)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("uplo", [1, 2], ids=["lower", "upper"])
def test_trsm_large_solve_with_1024_leaves(lib, dtype, uplo):
    """m = n = 4096 TRSM, the size from which the solve inverts 1024 x 1024
    diagonal blocks (one more doubling step) instead of 512 x 512.  12
    seeded columns of X against the long-double oracle solve of the same
    columns (relative forward error <= 4 * m * u on these well-conditioned
    systems), through device pointers; the same call through host pointers
    (column panels, each carrying the whole call's n) must be bit-identical."""
    torch = pytest.importorskip("torch")
    n, ncheck = 4096, 12
    dt = np.dtype(dtype)
    p = "s" if dt == np.float32 else "d"
    u = 2.0 ** -24 if p == "s" else 2.0 ** -53
    a = orc.trsm_matrix(n, dt, 5, 0)
    b = orc.fill(n, n, dt, 5, 1)
    sel = np.sort(np.random.default_rng(12).choice(n, ncheck, replace=False))
    ref = np.asfortranarray(b[:, sel])
    assert getattr(orc.restated(), f"oracle_{p}trsm")(0, uplo, 0, 0, n, ncheck, 1.0,
                                                     a.ctypes.data, 1, n, ref.ctypes.data, 1,
                                                     n) == 0
    fn = getattr(lib, f"mublis_{p}trsm")
    ad = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    x = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    assert fn(0, uplo, 0, 0, n, n, 1.0, ad.data_ptr(), 1, n, x.data_ptr(), 1, n) == 0, \
        mb.last_error(lib)
    dev = np.asfortranarray(x.cpu().numpy().T)
    got = dev[:, sel].astype(np.float64)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= 4 * n * u, err
    host = np.asfortranarray(b.copy())
    assert fn(0, uplo, 0, 0, n, n, 1.0, a.ctypes.data, 1, n, host.ctypes.data, 1, n) == 0, \
        mb.last_error(lib)
    np.testing.assert_array_equal(host, dev)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("m,n", [(16, 1), (17, 33), (511, 65), (513, 31), (1040, 100),
                                 (1537, 257)])
@pytest.mark.parametrize("flags", [dict(right=False, lower=True, ta=False, unit=False),
                                   dict(right=False, lower=False, ta=False, unit=True),
                                   dict(right=False, lower=True, ta=True, unit=False),
                                   dict(right=True, lower=False, ta=False, unit=False)],
                         ids=["LLN", "LUNu", "LLT", "RUN"])
def test_trsm_leaf_boundaries(lib, dtype, m, n, flags):
    """Solves whose order falls on and around the fused kernel's 16-row
    diagonal blocks and 512-row leaves, with right-hand-side counts around
    its 32-column CTAs, in both triangles, both layouts of op(A), unit and
    non-unit diagonals, and from the right: against the oracle (relative
    forward error <= 4 * order * u)."""
    case = dict(routine="trsm", dtype=dtype, order="F", m=m, n=n, k=0, alpha=0.75, seed=17,
                **flags)
    a, b, c0, out = run_lib(lib, case)
    ref = run_oracle(case)
    assert np.isfinite(out).all()
    assert cs.normwise_error(case, out, ref, a, b, c0) <= tol_of(case)
