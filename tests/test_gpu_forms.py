"""Precision forms on the tensor cores, against the oracle.

Stated tolerances (normwise relative error against the long-double oracle
restatement, or against a double-double evaluation of sampled entries at
8192^3):
  plain FP32 / FP64     4 * k * u                      (u = 2^-24 / 2^-53)
  bf16x6 (FP32)         4 * k * 2^-24                  (same as plain)
  bf16x3 (FP32)         2^-19   (the split keeps 16 bits of each input,
                                 |x - hi - lo| <= 2^-18 |x|; the error is
                                 not k-dependent, ~2^-18 / sqrt(k) normwise
                                 for random signs); at 8192^3 at most 4x
                                 plain FP32's measured error
  fp16x3 (FP32)         4 * k * 2^-24  (scaled fp16 split: ~24-bit inputs)
  ozaki:8 (FP64)        4 * k * 2^-53                  (same as plain)
  ozaki:7 (FP64)        2^-44
  ozaki2 (FP64, 16 moduli, ~55-bit inputs)   4 * k * 2^-53
  ozaki2 (FP32, 8 moduli, ~25-bit inputs)    4 * k * 2^-24
  ozaki2:14 (FP64, ~49-bit inputs at k=700)  2^-44
  ozaki2:6 (FP64, ~18-bit inputs: checks the CRT with M < 2^84)  2^-14
The 8192^3 study also checks the headline claims: bf16x6 has the error of
plain FP32 (within 1.5x), fp16x3 at most plain FP32's, and ozaki:8 and
ozaki2 at most the error of plain FP64.
Run with -s to print the measured table.
"""
import ctypes

import numpy as np
import pytest

import mublis_b200 as mb
from oracle import oracle as orc
from tests import cases as cs

pytestmark = pytest.mark.gpu

TOL = {
    "plain": lambda k, u: 4 * k * u,
    "bf16x6": lambda k, u: 4 * k * 2.0 ** -24,
    "fp16x3": lambda k, u: 4 * k * 2.0 ** -24,
    "bf16x3": lambda k, u: 2.0 ** -19,
    "ozaki:8": lambda k, u: 4 * k * 2.0 ** -53,
    "ozaki:7": lambda k, u: 2.0 ** -44,
    "ozaki2": lambda k, u: 4 * k * u,
    "ozaki2:14": lambda k, u: 2.0 ** -44,
    "ozaki2:6": lambda k, u: 2.0 ** -14,
}


@pytest.fixture(scope="module")
def lib():
    lib = mb.load()
    assert lib.mublis_b200_init() == 0, mb.last_error(lib)
    orc.set_threads(16)
    yield lib
    lib.mublis_b200_set_form(b"s", b"plain")
    lib.mublis_b200_set_form(b"d", b"plain")


def run(lib, case, form):
    p = b"s" if case["dtype"] == "float32" else b"d"
    assert lib.mublis_b200_set_form(p, form.encode()) == 0
    a, b, c0 = cs.build(case)
    out = c0.copy(order="K")
    cs.cblas_call(lib, case, a, b, out)
    ref = c0.copy(order="K")
    cs.oracle_call(case, a, b, ref)
    lib.mublis_b200_set_form(p, b"plain")
    return cs.normwise_error(case, out, ref, a, b, c0), np.isfinite(out[cs.active_mask(case)]).all()


FAMILY = [("gemm", dict(ta=False, tb=False)), ("gemm", dict(ta=True, tb=True)),
          ("symm", dict(right=False, lower=True)), ("symm", dict(right=True, lower=False)),
          ("syrk", dict(ta=False, lower=True)), ("syr2k", dict(ta=True, lower=False)),
          ("trmm", dict(right=False, lower=True, ta=False, unit=False)),
          ("trmm", dict(right=True, lower=False, ta=True, unit=True)),
          ("trsm", dict(right=False, lower=True, ta=False, unit=False))]


@pytest.mark.parametrize("form", ["bf16x3", "bf16x6", "fp16x3", "ozaki2"])
@pytest.mark.parametrize("routine,flags", FAMILY, ids=[f"{r}{i}" for i, (r, _) in enumerate(FAMILY)])
def test_fp32_tensor_forms(lib, form, routine, flags):
    case = dict(routine=routine, dtype="float32", order="F", m=640, n=544, k=704, alpha=0.75,
                beta=0.25, seed=21, **flags)
    if routine in ("syrk", "syr2k"):
        case["m"] = case["n"]
    err, finite = run(lib, case, form)
    assert finite
    assert err <= TOL[form](cs.inner_dim(case), 2.0 ** -24), err


@pytest.mark.parametrize("form", ["ozaki:7", "ozaki:8", "ozaki2", "ozaki2:14", "ozaki2:6"])
@pytest.mark.parametrize("routine,flags", FAMILY, ids=[f"{r}{i}" for i, (r, _) in enumerate(FAMILY)])
def test_fp64_ozaki(lib, form, routine, flags):
    case = dict(routine=routine, dtype="float64", order="F", m=600, n=520, k=680, alpha=0.75,
                beta=0.25, seed=22, **flags)
    if routine in ("syrk", "syr2k"):
        case["m"] = case["n"]
    err, finite = run(lib, case, form)
    assert finite
    assert err <= TOL[form](cs.inner_dim(case), 2.0 ** -53), err


def test_auto_form_matches_plain_error(lib):
    case = dict(routine="gemm", dtype="float32", order="F", m=1024, n=1024, k=1024, ta=False,
                tb=False, alpha=1.0, beta=0.5, seed=3)
    err, finite = run(lib, case, "auto")
    assert finite and err <= TOL["plain"](1024, 2.0 ** -24)


def test_auto_form_fp64_picks_emulation_within_plain_error(lib):
    """At 2048^3 "auto" runs FP64 GEMM on the modular form; its error against
    double-double values of 512 sampled entries must stay within plain's
    bound."""
    n = 2048
    a = orc.fill(n, n, np.float64, 12, 0)
    b = orc.fill(n, n, np.float64, 12, 1)
    c0 = orc.fill(n, n, np.float64, 12, 2)
    rng = np.random.default_rng(4)
    rows, cols = rng.integers(0, n, 512), rng.integers(0, n, 512)
    hi, lo = orc.dd_gemm_entries(a, b, rows, cols, alpha=1.0, beta=0.5, c0=c0)
    assert lib.mublis_b200_set_form(b"d", b"auto") == 0
    c = c0.copy(order="F")
    assert lib.mublis_dgemm(0, 0, n, n, n, 1.0, a.ctypes.data, 1, n, b.ctypes.data, 1, n, 0.5,
                            c.ctypes.data, 1, n) == 0, mb.last_error(lib)
    lib.mublis_b200_set_form(b"d", b"plain")
    d = c[rows, cols] - (hi + lo)
    den = np.linalg.norm(a) * np.linalg.norm(b) + 0.5 * np.linalg.norm(c0)
    err = np.sqrt((d ** 2).sum() * n * n / len(rows)) / den
    assert err <= 4 * n * 2.0 ** -53, err


def test_auto_form_fp32_large_is_fp16x3_within_plain_error(lib):
    """From 4096 on "auto" runs FP32 GEMM as fp16x3: the result is
    bit-identical to an explicit fp16x3 call, and its error against
    double-double values of 512 sampled entries is within plain's bound."""
    n = 4096
    a = orc.fill(n, n, np.float32, 13, 0)
    b = orc.fill(n, n, np.float32, 13, 1)
    c0 = orc.fill(n, n, np.float32, 13, 2)
    rng = np.random.default_rng(5)
    rows, cols = rng.integers(0, n, 512), rng.integers(0, n, 512)
    hi, lo = orc.dd_gemm_entries(a, b, rows, cols, alpha=1.0, beta=0.5, c0=c0)
    out = {}
    for form in ("auto", "fp16x3"):
        assert lib.mublis_b200_set_form(b"s", form.encode()) == 0
        c = c0.copy(order="F")
        assert lib.mublis_sgemm(0, 0, n, n, n, 1.0, a.ctypes.data, 1, n, b.ctypes.data, 1, n,
                                0.5, c.ctypes.data, 1, n) == 0, mb.last_error(lib)
        out[form] = c
    lib.mublis_b200_set_form(b"s", b"plain")
    np.testing.assert_array_equal(out["auto"], out["fp16x3"])
    d = out["auto"][rows, cols].astype(np.float64) - (hi + lo)
    den = np.linalg.norm(a.astype(np.float64)) * np.linalg.norm(b.astype(np.float64)) + \
        0.5 * np.linalg.norm(c0.astype(np.float64))
    err = np.sqrt((d ** 2).sum() * n * n / len(rows)) / den
    assert err <= 4 * n * 2.0 ** -24, err


def test_wide_range_inputs_ozaki(lib):
    """The wide draw (|x| = m * 2^e, e in [-10, 10]) stresses the per-row
    scaling of the Ozaki split."""
    torch = pytest.importorskip("torch")
    n = 1536
    a = orc.fill(n, n, np.float64, 4, 0, orc.WIDE)
    b = orc.fill(n, n, np.float64, 4, 1, orc.WIDE)
    rows = np.random.default_rng(0).integers(0, n, 512)
    cols = np.random.default_rng(1).integers(0, n, 512)
    hi, lo = orc.dd_gemm_entries(a, b, rows, cols)
    exact = hi + lo
    den = np.linalg.norm(a) * np.linalg.norm(b)
    errs = {}
    for form in ("plain", "ozaki:8", "ozaki2"):
        assert lib.mublis_b200_set_form(b"d", form.encode()) == 0
        c = np.zeros((n, n), order="F")
        assert lib.mublis_dgemm(0, 0, n, n, n, 1.0, a.ctypes.data, 1, n, b.ctypes.data, 1, n,
                                0.0, c.ctypes.data, 1, n) == 0
        d = c[rows, cols] - exact
        errs[form] = np.sqrt((d ** 2).sum() * n * n / len(rows)) / den
    lib.mublis_b200_set_form(b"d", b"plain")
    assert errs["ozaki:8"] <= max(errs["plain"], 4 * n * 2.0 ** -53), errs
    assert errs["ozaki2"] <= max(errs["plain"], 4 * n * 2.0 ** -53), errs


@pytest.mark.parametrize("form", ["ozaki:8", "ozaki2"])
def test_ozaki_long_k_chunks(lib, form):
    """k = 70001 spans several exact-int32 chunks of both integer forms
    (8192 for slices, 32768 for moduli): the per-chunk partial results must
    combine to the double-double value of sampled entries."""
    m, n, k = 200, 136, 70001
    a = orc.fill(m, k, np.float64, 9, 0)
    b = orc.fill(k, n, np.float64, 9, 1)
    c0 = orc.fill(m, n, np.float64, 9, 2)
    rng = np.random.default_rng(5)
    rows, cols = rng.integers(0, m, 256), rng.integers(0, n, 256)
    hi, lo = orc.dd_gemm_entries(a, b, rows, cols, alpha=0.75, beta=0.25, c0=c0)
    assert lib.mublis_b200_set_form(b"d", form.encode()) == 0
    c = c0.copy(order="F")
    assert lib.mublis_dgemm(0, 0, m, n, k, 0.75, a.ctypes.data, 1, m, b.ctypes.data, 1, k,
                            0.25, c.ctypes.data, 1, m) == 0, mb.last_error(lib)
    lib.mublis_b200_set_form(b"d", b"plain")
    d = c[rows, cols] - (hi + lo)
    den = 0.75 * np.linalg.norm(a) * np.linalg.norm(b) + 0.25 * np.linalg.norm(c0)
    err = np.sqrt((d ** 2).sum() * m * n / len(rows)) / den
    assert err <= 4 * k * 2.0 ** -53, err


def _device_matrix(torch, lib, p, n, seed, mid, kind=0):
    dt = torch.float32 if p == "s" else torch.float64
    t = torch.empty(n, n, dtype=dt, device="cuda")
    fill = getattr(lib, f"mublis_b200_fill_{p}")
    assert fill(ctypes.c_void_p(t.data_ptr()), n, n, n, seed, mid, kind) == 0
    return t


def _full_lines(n, lines, seed):
    """Entry indices of `lines`/2 full rows and `lines`/2 full columns of an
    n x n matrix (seeded choice)."""
    rng = np.random.default_rng(seed)
    r_sel = rng.choice(n, lines // 2, replace=False)
    c_sel = rng.choice(n, lines // 2, replace=False)
    rows = np.concatenate([np.repeat(r_sel, n), np.tile(np.arange(n), len(c_sel))])
    cols = np.concatenate([np.tile(np.arange(n), len(r_sel)), np.repeat(c_sel, n)])
    return rows, cols


@pytest.mark.parametrize("kind", [orc.UNIFORM, orc.WIDE], ids=["uniform", "wide"])
def test_precision_study_8192(lib, kind):
    """Config-3 study: m = n = k = 8192, uniform and wide draws; normwise and
    max elementwise error of every form against double-double values of
    128 full rows and 128 full columns of alpha*A*B + beta*C (alpha 1,
    beta 0.5).  The normwise figure is the sampled Frobenius norm scaled to
    the whole matrix."""
    torch = pytest.importorskip("torch")
    n = 8192
    rows, cols = _full_lines(n, 256, 7)
    ns = len(rows)
    table = {}
    for p, forms in (("s", ["plain", "bf16x3", "bf16x6", "fp16x3", "ozaki2"]),
                     ("d", ["plain", "ozaki:7", "ozaki:8", "ozaki2:14", "ozaki2"])):
        a, b, c0 = (_device_matrix(torch, lib, p, n, 0, i, kind) for i in range(3))
        # torch holds the column-major matrices transposed: a.cpu() is A^T in
        # row-major order, i.e. a column-major A^T, so op(A) = (A^T)^T reads
        # both operands contiguously in the double-double oracle.
        at = np.asfortranarray(a.cpu().numpy())
        bh, ch = (np.asfortranarray(x.cpu().numpy().T) for x in (b, c0))
        hi, lo = orc.dd_gemm_entries(at, bh, rows, cols, alpha=1.0, beta=0.5, c0=ch, ta=True)
        exact = hi + lo
        den = (np.linalg.norm(at.astype(np.float64)) * np.linalg.norm(bh.astype(np.float64)) +
               0.5 * np.linalg.norm(ch.astype(np.float64)))
        del at, bh, ch
        fn = getattr(lib, f"mublis_{p}gemm")
        for form in forms:
            assert lib.mublis_b200_set_form(p.encode(), form.encode()) == 0
            c = c0.clone()
            torch.cuda.synchronize()
            assert fn(0, 0, n, n, n, 1.0, a.data_ptr(), 1, n, b.data_ptr(), 1, n, 0.5,
                      c.data_ptr(), 1, n) == 0
            got = c.cpu().numpy().T[rows, cols].astype(np.float64)
            d = got - exact
            nw = np.sqrt((d ** 2).sum() * (n * n / ns)) / den
            mx = float(np.max(np.abs(d) / np.maximum(np.abs(exact), 1e-300)))
            table[f"{p}gemm {form}"] = (nw, mx)
        lib.mublis_b200_set_form(p.encode(), b"plain")
        del a, b, c0
        torch.cuda.empty_cache()
    print(f"\nm=n=k=8192, draw={'wide' if kind else 'uniform'}, 128 full rows + 128 full "
          "columns: normwise, max elementwise rel")
    for key, (nw, mx) in table.items():
        print(f"  {key:16s} {nw:.3e}  {mx:.3e}")
    assert table["sgemm bf16x6"][0] <= 1.5 * table["sgemm plain"][0]
    assert table["dgemm ozaki:8"][0] <= table["dgemm plain"][0]
    assert table["dgemm ozaki2"][0] <= table["dgemm plain"][0]
    assert table["sgemm ozaki2"][0] <= table["sgemm plain"][0]
    assert table["sgemm fp16x3"][0] <= table["sgemm plain"][0]
    assert table["sgemm bf16x3"][0] <= 4 * table["sgemm plain"][0]
    assert table["dgemm ozaki:7"][0] <= TOL["ozaki:7"](n, 0)


def test_dtrsm_8192_forms(lib):
    """Config-3 DTRSM: n = 8192 with 8192 right-hand sides (left, lower,
    non-unit, A well conditioned), plain against the emulated off-diagonal
    updates (the diagonal blocks stay FP64).  16 seeded columns of X are
    checked against the long-double oracle solve of the same columns."""
    torch = pytest.importorskip("torch")
    n, ncheck = 8192, 16
    a = orc.trsm_matrix(n, np.float64, 3, 0)
    b = orc.fill(n, n, np.float64, 3, 1)
    sel = np.sort(np.random.default_rng(11).choice(n, ncheck, replace=False))
    ref = np.asfortranarray(b[:, sel])
    orc.set_threads(16)
    assert orc.restated().oracle_dtrsm(0, 1, 0, 0, n, ncheck, 1.0, a.ctypes.data, 1, n,
                                       ref.ctypes.data, 1, n) == 0
    ad = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    b0 = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    errs = {}
    for form in ("plain", "ozaki2"):
        assert lib.mublis_b200_set_form(b"d", form.encode()) == 0
        x = b0.clone()
        assert lib.mublis_dtrsm(0, 1, 0, 0, n, n, 1.0, ad.data_ptr(), 1, n, x.data_ptr(), 1,
                                n) == 0, mb.last_error(lib)
        got = x.cpu().numpy().T[:, sel]
        d = got - ref
        errs[form] = (np.linalg.norm(d) / np.linalg.norm(ref),
                      float(np.max(np.abs(d) / np.maximum(np.abs(ref), 1e-300))))
    lib.mublis_b200_set_form(b"d", b"plain")
    print(f"\nDTRSM n=8192, 8192 RHS, {ncheck} columns checked: normwise, max elementwise rel")
    for form, (nw, mx) in errs.items():
        print(f"  dtrsm {form:8s} {nw:.3e}  {mx:.3e}")
    assert errs["plain"][0] <= 4 * n * 2.0 ** -53
    assert errs["ozaki2"][0] <= 4 * n * 2.0 ** -53


@pytest.mark.parametrize("kind", [orc.UNIFORM, orc.WIDE], ids=["uniform", "wide"])
def test_ozaki2_autotune_picks_fewest_moduli_for_target(lib, kind):
    """mublis_b200_ozaki2_autotune (the modulus count chosen for a
    stated error): a looser target never takes more moduli than a tighter
    one, the measured calibration error of the choice meets the target
    (unless all 16 moduli were needed), and a call with form
    "ozaki2@<target>" then meets the target on the whole product, against
    double-double values of 512 sampled entries (within 2x: the choice was
    measured on the leading 256 x 256 block)."""
    torch = pytest.importorskip("torch")
    n = 2048
    a = orc.fill(n, n, np.float64, 14, 0, kind)
    b = orc.fill(n, n, np.float64, 14, 1, kind)
    ad = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    bd = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    rng = np.random.default_rng(6)
    rows, cols = rng.integers(0, n, 512), rng.integers(0, n, 512)
    hi, lo = orc.dd_gemm_entries(a, b, rows, cols)
    den = np.linalg.norm(a) * np.linalg.norm(b)
    chosen = []
    for target in (1e-13, 1e-15, 1e-17):
        nm, err = ctypes.c_int(), ctypes.c_double()
        assert lib.mublis_b200_ozaki2_autotune(b"d", 0, 0, n, n, n, ad.data_ptr(), 1, n,
                                               bd.data_ptr(), 1, n, target, ctypes.byref(nm),
                                               ctypes.byref(err)) == 0, mb.last_error(lib)
        assert 6 <= nm.value <= 16
        assert err.value <= target or nm.value == 16, (target, nm.value, err.value)
        chosen.append(nm.value)
        assert lib.mublis_b200_set_form(b"d", f"ozaki2@{target!r}".encode()) == 0
        c = torch.zeros(n, n, dtype=torch.float64, device="cuda")
        assert lib.mublis_dgemm(0, 0, n, n, n, 1.0, ad.data_ptr(), 1, n, bd.data_ptr(), 1, n,
                                0.0, c.data_ptr(), 1, n) == 0, mb.last_error(lib)
        lib.mublis_b200_set_form(b"d", b"plain")
        d = c.cpu().numpy().T[rows, cols] - (hi + lo)
        whole = np.sqrt((d ** 2).sum() * n * n / len(rows)) / den
        if nm.value < 16:
            assert whole <= 2 * target, (target, nm.value, whole)
    print(f"\nozaki2 autotune, n=2048, draw={'wide' if kind else 'uniform'}: "
          f"targets 1e-13/1e-15/1e-17 -> {chosen} moduli")
    assert chosen == sorted(chosen)


def test_ozaki2_autotune_fp32(lib):
    """FP32 inputs: a target at plain FP32's level is met with at most the
    default 8 moduli."""
    torch = pytest.importorskip("torch")
    n = 1024
    a = torch.empty(n, n, dtype=torch.float32, device="cuda")
    b = torch.empty(n, n, dtype=torch.float32, device="cuda")
    lib.mublis_b200_fill_s(ctypes.c_void_p(a.data_ptr()), n, n, n, 15, 0, 0)
    lib.mublis_b200_fill_s(ctypes.c_void_p(b.data_ptr()), n, n, n, 15, 1, 0)
    nm, err = ctypes.c_int(), ctypes.c_double()
    assert lib.mublis_b200_ozaki2_autotune(b"s", 0, 0, n, n, n, a.data_ptr(), 1, n, b.data_ptr(),
                                           1, n, 1e-7, ctypes.byref(nm),
                                           ctypes.byref(err)) == 0, mb.last_error(lib)
    assert 6 <= nm.value <= 8 and err.value <= 1e-7, (nm.value, err.value)
