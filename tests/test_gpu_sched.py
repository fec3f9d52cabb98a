"""The device tile scheduler's split-K path and the FP64 kernel's direct
operand loads, against the oracle (GPU).

Split-K (sched.cu) runs only where the whole call has too few tiles for its
k; these shapes are chosen to take it: SYRK with n = 1024, k = 8192 (36
lower-triangle tiles), GEMM 1024^3 (64 tiles of 128 x 128), a k-dominant
GEMM 256 x 256 x 8192, and a TRMM whose tiles' k ranges are clipped (pi).
Each result is checked against the long-double oracle on seeded columns
(normwise relative error <= 4 k u), and, through host pointers (the
pipelined staging path cuts C into column panels), must be bit-identical to
the device-pointer result: the split count depends only on the whole call.

Direct loads (the FP64 tensor-pipe kernel reading op(A) / op(B) as 2-D TMA
tiles, no pack pass) run for device operands with an even leading dimension
and a 16-byte aligned base: ragged sizes in all four transposes (the TMA
tiles' out-of-range rows and k fill with zeros), row-major operands (k as
the unit stride: swizzled tiles), SYR2K with k a multiple of 16 (two tensor
maps split at the pair boundary) and not (packed instead), and a base
offset by one element (8-byte aligned: packed instead) -- all against the
oracle within 4 k u.
"""
import numpy as np
import pytest

import mublis_b200 as mb
from oracle import oracle as orc
from tests import cases as cs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = mb.load()
    assert lib.mublis_b200_init() == 0, mb.last_error(lib)
    lib.mublis_b200_set_form(b"s", b"plain")
    lib.mublis_b200_set_form(b"d", b"plain")
    orc.set_threads(16)
    return lib


def to_dev(torch, x):
    """Column-major numpy array -> device tensor holding the same bytes."""
    return torch.from_numpy(np.asfortranarray(x).T.copy()).cuda()


def from_dev(t):
    return np.asfortranarray(t.cpu().numpy().T)


def bits(x):
    return x.view(np.uint32 if x.dtype == np.float32 else np.uint64)


SPLIT_CASES = [
    dict(routine="syrk", m=1024, n=1024, k=8192, ta=False, lower=True),
    dict(routine="gemm", m=1024, n=1024, k=1024, ta=False, tb=False),
    dict(routine="gemm", m=256, n=256, k=8192, ta=True, tb=False),
    dict(routine="trmm", m=512, n=96, k=0, right=False, lower=True, ta=False, unit=False),
]


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("sc", SPLIT_CASES, ids=[f"{c['routine']}{c['m']}x{c['n']}x{c['k']}"
                                                 for c in SPLIT_CASES])
def test_split_k_shapes_match_oracle_and_host_bits(lib, dtype, sc):
    torch = pytest.importorskip("torch")
    case = dict(dtype=dtype, order="F", alpha=0.75, beta=0.25, seed=23, **sc)
    if case["routine"] == "trsm":
        case.pop("beta")
    a, b, c0 = cs.build(case)
    # device pointers
    out_dev_t = to_dev(torch, c0)
    da = to_dev(torch, a)
    db = None if b is None else to_dev(torch, b)
    torch.cuda.synchronize()
    p = "s" if dtype == "float32" else "d"
    fn = getattr(lib, f"cblas_{p}{case['routine']}")
    r = case["routine"]
    M, N, K = case["m"], case["n"], case["k"]
    if r == "gemm":
        lda = K if case["ta"] else M
        ldb = N if case["tb"] else K
        fn(mb.COL, mb.TRANS if case["ta"] else mb.NO_TRANS, mb.TRANS if case["tb"] else mb.NO_TRANS,
           M, N, K, 0.75, da.data_ptr(), lda, db.data_ptr(), ldb, 0.25, out_dev_t.data_ptr(), M)
    elif r == "syrk":
        fn(mb.COL, mb.LOWER, mb.NO_TRANS, N, K, 0.75, da.data_ptr(), N, 0.25,
           out_dev_t.data_ptr(), N)
    else:  # trmm: c0 is B
        fn(mb.COL, mb.LEFT, mb.LOWER, mb.NO_TRANS, mb.NON_UNIT, M, N, 0.75, da.data_ptr(), M,
           out_dev_t.data_ptr(), M)
    torch.cuda.synchronize()
    out_dev = from_dev(out_dev_t)
    ref = c0.copy(order="F")
    cs.oracle_call(case, a, b, ref)
    mask = cs.active_mask(case)
    assert np.isfinite(out_dev[mask]).all()
    err = cs.normwise_error(case, out_dev, ref, a, b, c0)
    assert err <= 4 * max(cs.inner_dim(case), 1) * cs.EPS[np.dtype(dtype)], err
    # host pointers: bit-identical
    out_host = c0.copy(order="F")
    cs.cblas_call(lib, case, a, b, out_host)
    np.testing.assert_array_equal(bits(out_host), bits(out_dev))


def padded(x, extra_rows):
    """x (column-major) inside a larger column-major buffer whose leading
    dimension is rows + extra_rows; returns (buffer, view)."""
    buf = np.zeros((x.shape[0] + extra_rows, x.shape[1]), dtype=x.dtype, order="F")
    buf[:x.shape[0], :] = x
    return buf


@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("mnk", [(127, 129, 255), (300, 200, 513), (1, 255, 128), (257, 130, 16),
                                 (129, 1, 300)])
def test_direct_loads_ragged_even_ld(lib, ta, tb, mnk):
    """FP64 GEMM from device operands whose leading dimensions are even
    (TMA-eligible) at ragged sizes: edge tiles, partial k-blocks."""
    torch = pytest.importorskip("torch")
    m, n, k = mnk
    case = dict(routine="gemm", dtype="float64", order="F", m=m, n=n, k=k, ta=ta, tb=tb,
                alpha=0.75, beta=0.25, seed=24)
    a, b, c0 = cs.build(case)
    abuf = padded(a, a.shape[0] % 2)   # even leading dimension
    bbuf = padded(b, b.shape[0] % 2)
    da, db, dc = to_dev(torch, abuf), to_dev(torch, bbuf), to_dev(torch, c0)
    torch.cuda.synchronize()
    assert lib.mublis_dgemm(int(ta), int(tb), m, n, k, 0.75, da.data_ptr(), 1, abuf.shape[0],
                            db.data_ptr(), 1, bbuf.shape[0], 0.25, dc.data_ptr(), 1, m) == 0, \
        mb.last_error(lib)
    torch.cuda.synchronize()
    out = from_dev(dc)
    ref = c0.copy(order="F")
    cs.oracle_call(case, a, b, ref)
    assert cs.normwise_error(case, out, ref, a, b, c0) <= 4 * k * 2.0 ** -53


@pytest.mark.parametrize("ta", [False, True])
def test_direct_loads_row_major(lib, ta):
    """Row-major operands through cblas (k as the unit stride of op(A) /
    op(B) in one of them: swizzled tiles)."""
    torch = pytest.importorskip("torch")
    m, n, k = 200, 190, 330
    case = dict(routine="gemm", dtype="float64", order="C", m=m, n=n, k=k, ta=ta, tb=not ta,
                alpha=0.75, beta=0.25, seed=25)
    a, b, c0 = cs.build(case)
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    dc = torch.from_numpy(np.ascontiguousarray(c0)).cuda()
    torch.cuda.synchronize()
    lib.cblas_dgemm(mb.ROW, mb.TRANS if ta else mb.NO_TRANS, mb.NO_TRANS if ta else mb.TRANS,
                    m, n, k, 0.75, da.data_ptr(), a.shape[1], db.data_ptr(), b.shape[1], 0.25,
                    dc.data_ptr(), n)
    torch.cuda.synchronize()
    out = dc.cpu().numpy()
    ref = c0.copy()
    cs.oracle_call(case, a, b, ref)
    assert cs.normwise_error(case, out, ref, a, b, c0) <= 4 * k * 2.0 ** -53


@pytest.mark.parametrize("k", [256, 250])
def test_direct_loads_syr2k_pairs(lib, k):
    """SYR2K's two pairs: direct with two tensor maps when k is a multiple of
    16, packed otherwise; both against the oracle."""
    torch = pytest.importorskip("torch")
    n = 300
    case = dict(routine="syr2k", dtype="float64", order="F", m=n, n=n, k=k, ta=False, lower=True,
                alpha=0.75, beta=0.25, seed=26)
    a, b, c0 = cs.build(case)
    da, db, dc = to_dev(torch, a), to_dev(torch, b), to_dev(torch, c0)
    torch.cuda.synchronize()
    lib.cblas_dsyr2k(mb.COL, mb.LOWER, mb.NO_TRANS, n, k, 0.75, da.data_ptr(), n, db.data_ptr(),
                     n, 0.25, dc.data_ptr(), n)
    torch.cuda.synchronize()
    out = from_dev(dc)
    ref = c0.copy(order="F")
    cs.oracle_call(case, a, b, ref)
    mask = cs.active_mask(case)
    assert cs.normwise_error(case, out, ref, a, b, c0) <= 4 * 2 * k * 2.0 ** -53
    np.testing.assert_array_equal(out[~mask], c0[~mask])


def test_direct_loads_misaligned_base_falls_back(lib):
    """A base 8 bytes past a 16-byte boundary is not a TMA source: the
    operand is packed, and the result is the same as from an aligned copy."""
    torch = pytest.importorskip("torch")
    m, n, k = 160, 140, 96
    case = dict(routine="gemm", dtype="float64", order="F", m=m, n=n, k=k, ta=False, tb=False,
                alpha=0.75, beta=0.25, seed=27)
    a, b, c0 = cs.build(case)
    flat = torch.zeros(m * k + 1, dtype=torch.float64, device="cuda")
    flat[1:].copy_(torch.from_numpy(np.asfortranarray(a).T.reshape(-1).copy()))
    db, dc = to_dev(torch, b), to_dev(torch, c0)
    dc2 = dc.clone()
    da_al = to_dev(torch, a)
    torch.cuda.synchronize()
    assert lib.mublis_dgemm(0, 0, m, n, k, 0.75, flat.data_ptr() + 8, 1, m, db.data_ptr(), 1, k,
                            0.25, dc.data_ptr(), 1, m) == 0, mb.last_error(lib)
    assert lib.mublis_dgemm(0, 0, m, n, k, 0.75, da_al.data_ptr(), 1, m, db.data_ptr(), 1, k,
                            0.25, dc2.data_ptr(), 1, m) == 0, mb.last_error(lib)
    torch.cuda.synchronize()
    ref = c0.copy(order="F")
    cs.oracle_call(case, a, b, ref)
    assert cs.normwise_error(case, from_dev(dc), ref, a, b, c0) <= 4 * k * 2.0 ** -53
    np.testing.assert_array_equal(from_dev(dc), from_dev(dc2))
