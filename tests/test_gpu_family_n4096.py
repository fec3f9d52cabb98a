"""Parity of the benchmarked workload itself: the plain Level-3 family at
n = 4096 in FP32 and FP64, the 18 calls bench.py times, with its seeds.

Each call (cblas_*, column-major, alpha 0.75, beta 0.25):
  GEMM NN / NT / TN / TT at m = n = k = 4096; SYMM left/lower; SYRK and
  SYR2K lower, no-trans, n = k = 4096; TRMM and TRSM left/lower/non-unit
  with A = off-diagonals uniform[-1,1)/n, diagonal uniform[1,2);
  inputs seeded Philox uniform[-1,1), seed 0, matrix ids 3c + {0, 1, 2}
  for call c (the benchmark's ids).
Unstored triangles are NaN-poisoned as in the reference's own tests
(test/correctness/check_cblas.py:192-222): the upper triangle of SYMM's,
TRMM's and TRSM's A and of SYRK's / SYR2K's C.

Checked, through device pointers:
  * 16 seeded columns of the output (and, for GEMM, 16 seeded rows) against
    the long-double oracle restatement evaluated on the same columns (rows)
    in FP64, normwise relative error <= 4 * k * u (u = 2^-24 / 2^-53; k the
    inner dimension, 2n for SYR2K); TRSM: relative forward error
    <= 4 * n * u on these well-conditioned systems;
  * every written element finite; SYRK/SYR2K's upper triangle bit-identical
    to its (NaN) input.
And through host pointers (the pipelined staging path): the whole output
bit-identical to the device-pointer result.
"""
import numpy as np
import pytest

import mublis_b200 as mb
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N = 4096
NCHECK = 16
ALPHA, BETA = 0.75, 0.25
ROUTINES = ["gemm_nn", "gemm_nt", "gemm_tn", "gemm_tt", "symm", "syrk", "syr2k", "trmm", "trsm"]
CALLS = [(p, r, 3 * (9 * i + j)) for i, p in enumerate("sd") for j, r in enumerate(ROUTINES)]
COL, NT, TR, LOWER, NONUNIT, LEFT = 102, 111, 112, 122, 131, 141


@pytest.fixture(scope="module")
def lib():
    lib = mb.load()
    assert lib.mublis_b200_init() == 0, mb.last_error(lib)
    lib.mublis_b200_set_form(b"s", b"plain")
    lib.mublis_b200_set_form(b"d", b"plain")
    orc.set_threads(16)
    return lib


def inputs(p, r, mid):
    """(A, B, C0) as the benchmark builds them (C0 None for TRMM/TRSM, whose
    B is the in/out operand), column-major, unstored triangles NaN."""
    dt = np.float32 if p == "s" else np.float64
    upper = np.triu_indices(N, 1)
    if r in ("trmm", "trsm"):
        a = orc.trsm_matrix(N, dt, 0, mid)
    else:
        a = orc.fill(N, N, dt, 0, mid)
    if r in ("symm", "trmm", "trsm"):
        a[upper] = np.nan
    b = orc.fill(N, N, dt, 0, mid + 1)
    c0 = None
    if r not in ("trmm", "trsm"):
        c0 = orc.fill(N, N, dt, 0, mid + 2)
        if r in ("syrk", "syr2k"):
            c0[upper] = np.nan
    return a, b, c0


def call(lib, p, r, a, b, c):
    """One cblas_* call of the family; a, b, c are device (int) or host
    (numpy) pointers of column-major N x N operands."""
    fn = getattr(lib, f"cblas_{p}{r[:4] if r.startswith('gemm') else r}")
    if r.startswith("gemm"):
        ta = TR if r[5] == "t" else NT
        tb = TR if r[6] == "t" else NT
        fn(COL, ta, tb, N, N, N, ALPHA, a, N, b, N, BETA, c, N)
    elif r == "symm":
        fn(COL, LEFT, LOWER, N, N, ALPHA, a, N, b, N, BETA, c, N)
    elif r == "syrk":
        fn(COL, LOWER, NT, N, N, ALPHA, a, N, BETA, c, N)
    elif r == "syr2k":
        fn(COL, LOWER, NT, N, N, ALPHA, a, N, b, N, BETA, c, N)
    else:
        fn(COL, LEFT, LOWER, NT, NONUNIT, N, N, ALPHA, a, N, b, N)


def device_run(torch, lib, p, r, a, b, c0):
    """The call through device pointers; returns the output, column-major."""
    dev = [None if x is None else torch.from_numpy(np.asfortranarray(x).T).cuda()
           for x in (a, b, c0)]
    torch.cuda.synchronize()
    ptr = [None if x is None else x.data_ptr() for x in dev]
    call(lib, p, r, ptr[0], ptr[1], ptr[2])
    torch.cuda.synchronize()
    out = dev[1] if r in ("trmm", "trsm") else dev[2]
    return np.asfortranarray(out.cpu().numpy().T)


def bits(x):
    return x.view(np.uint32 if x.dtype == np.float32 else np.uint64)


def oracle_gemm(ta, tb, m, n, k, alpha, a, b, beta, c):
    """alpha op(a) op(b) + beta c by the long-double restatement, in FP64
    (inputs converted exactly); c is updated and returned."""
    a, b = np.asfortranarray(a, np.float64), np.asfortranarray(b, np.float64)
    c = np.asfortranarray(c, np.float64)
    assert orc.restated().oracle_dgemm(int(ta), int(tb), m, n, k, alpha, a.ctypes.data, 1,
                                       a.shape[0], b.ctypes.data, 1, b.shape[0], beta,
                                       c.ctypes.data, 1, c.shape[0]) == 0
    return c


def check_columns(p, r, a, b, c0, out, sel):
    """Normwise error of out[:, sel] (over the written part) divided by its
    bound."""
    u = 2.0 ** -24 if p == "s" else 2.0 ** -53
    j = len(sel)
    f64 = lambda x: np.asarray(x, np.float64)  # noqa: E731
    got = f64(out[:, sel])
    lower = np.arange(N)[:, None] >= sel[None, :]
    if r.startswith("gemm"):
        ta, tb = r[5] == "t", r[6] == "t"
        opb_cols = b[sel, :] if tb else b[:, sel]            # passed with tb
        ref = oracle_gemm(ta, tb, N, j, N, ALPHA, a, opb_cols, BETA, c0[:, sel])
        opa = f64(a).T if ta else f64(a)
        opb = f64(b[sel, :]).T if tb else f64(b[:, sel])
        den = ALPHA * np.linalg.norm(opa) * np.linalg.norm(opb) + BETA * np.linalg.norm(
            f64(c0[:, sel]))
        return np.linalg.norm(got - ref) / den / (4 * N * u)
    if r == "symm":
        ref = np.asfortranarray(c0[:, sel], np.float64)
        a64 = np.asfortranarray(a, np.float64)
        bs = np.asfortranarray(b[:, sel], np.float64)
        assert orc.restated().oracle_dsymm(0, 1, N, j, ALPHA, a64.ctypes.data, 1, N,
                                           bs.ctypes.data, 1, N, BETA, ref.ctypes.data, 1,
                                           N) == 0
        lo = np.tril(np.nan_to_num(f64(a)))
        sym = lo + np.tril(lo, -1).T
        den = ALPHA * np.linalg.norm(sym) * np.linalg.norm(bs) + BETA * np.linalg.norm(
            f64(c0[:, sel]))
        return np.linalg.norm(got - ref) / den / (4 * N * u)
    if r in ("syrk", "syr2k"):
        c0s = np.where(lower, f64(c0[:, sel]), 0.0)
        if r == "syrk":
            ref = oracle_gemm(False, True, N, j, N, ALPHA, a, a[sel, :], BETA, c0s)
            fa = np.linalg.norm(f64(a)) * np.linalg.norm(f64(a[sel, :]))
        else:
            ref = oracle_gemm(False, True, N, j, N, ALPHA, a, b[sel, :], BETA, c0s)
            ref = oracle_gemm(False, True, N, j, N, ALPHA, b, a[sel, :], 1.0, ref)
            fa = (np.linalg.norm(f64(a)) * np.linalg.norm(f64(b[sel, :])) +
                  np.linalg.norm(f64(b)) * np.linalg.norm(f64(a[sel, :])))
        diff = np.where(lower, got - ref, 0.0)
        den = ALPHA * fa + BETA * np.linalg.norm(c0s)
        k = 2 * N if r == "syr2k" else N
        return np.linalg.norm(diff) / den / (4 * k * u)
    # TRMM / TRSM: b is the input right-hand side
    a64 = np.asfortranarray(a, np.float64)
    ref = np.asfortranarray(b[:, sel], np.float64)
    fn = orc.restated().oracle_dtrmm if r == "trmm" else orc.restated().oracle_dtrsm
    assert fn(0, 1, 0, 0, N, j, ALPHA, a64.ctypes.data, 1, N, ref.ctypes.data, 1, N) == 0
    if r == "trmm":
        den = ALPHA * np.linalg.norm(np.tril(np.nan_to_num(a64))) * np.linalg.norm(
            f64(b[:, sel]))
    else:
        den = np.linalg.norm(ref)
    return np.linalg.norm(got - ref) / den / (4 * N * u)


@pytest.mark.parametrize("p,r,mid", CALLS, ids=[f"{p}{r}" for p, r, _ in CALLS])
def test_benchmarked_call_at_n4096(lib, p, r, mid):
    torch = pytest.importorskip("torch")
    a, b, c0 = inputs(p, r, mid)
    out = device_run(torch, lib, p, r, a, b, c0)
    written = np.tril(np.ones((N, N), bool)) if r in ("syrk", "syr2k") else np.ones((N, N), bool)
    assert np.isfinite(out[written]).all()
    if r in ("syrk", "syr2k"):
        np.testing.assert_array_equal(bits(out[~written]), bits(c0[~written]))

    rng = np.random.default_rng(1000 + mid)
    sel = np.sort(rng.choice(N, NCHECK, replace=False))
    ratio = check_columns(p, r, a, b, c0, out, sel)
    assert ratio <= 1.0, f"{p}{r}: columns error / bound = {ratio}"
    if r.startswith("gemm"):
        # Rows: C[sel, :] = alpha op(A)[sel, :] op(B) + beta C0[sel, :].
        ta, tb = r[5] == "t", r[6] == "t"
        u = 2.0 ** -24 if p == "s" else 2.0 ** -53
        opa_rows = a[:, sel] if ta else a[sel, :]
        ref = oracle_gemm(ta, tb, NCHECK, N, N, ALPHA, opa_rows, b, BETA, c0[sel, :])
        f64 = lambda x: np.asarray(x, np.float64)  # noqa: E731
        den = ALPHA * np.linalg.norm(f64(opa_rows)) * np.linalg.norm(f64(b)) + \
            BETA * np.linalg.norm(f64(c0[sel, :]))
        err = np.linalg.norm(f64(out[sel, :]) - ref) / den
        assert err <= 4 * N * u, f"{p}{r}: rows error {err}"

    # Host pointers: the pipelined staging path gives the device call's bits.
    host_out = (b if r in ("trmm", "trsm") else c0).copy(order="F")
    hb = host_out if r in ("trmm", "trsm") else b
    call(lib, p, r, a.ctypes.data, None if hb is None else hb.ctypes.data,
         None if r in ("trmm", "trsm") else host_out.ctypes.data)
    np.testing.assert_array_equal(bits(host_out), bits(out))
