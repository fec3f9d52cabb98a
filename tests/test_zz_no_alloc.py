"""mublis_b200_sgemm_noalloc: the SGEMM entry point that allocates nothing.

It exists for callers that cannot allocate device memory when they call in:
processes whose GPU memory is already owned by another allocator, or services
that keep a fixed device footprint and ban cudaMalloc/cudaFree on their
request path.  Instead of per-call scratch it packs operands into a fixed
32 MiB array in the library's device code, claimed when the library
initialises.

Checked here, through the C ABI:
  * two calls in a row (different shapes, transposes and inputs, so the
    second call runs over the first call's leftover scratch contents) agree
    with mublis_sgemm on the same device operands within the suite's
    tolerance (normwise relative error <= 4 * k * 2^-24);
  * neither call takes memory: the used-memory high watermark of the
    device's default stream-ordered pool (where the library's scratch comes
    from) stays at its value before the call, and the device's free memory
    is unchanged;
  * the size limit is exact: m = n = k = 2048 (exactly the limit) runs and
    matches mublis_sgemm, k = 2049 (one more k block) and 4096^3 are refused
    with a clear error and leave C untouched;
  * empty sizes return before the sizes are checked, as mublis_sgemm does.

This file is named to be collected last, so a failure here comes after every
other test has run; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import mublis_b200 as mb

pytestmark = pytest.mark.gpu

CU_MEMPOOL_ATTR_USED_MEM_CURRENT = 7
CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8


@pytest.fixture(scope="module")
def lib():
    lib = mb.load()
    assert lib.mublis_b200_init() == 0, mb.last_error(lib)
    lib.mublis_b200_set_form(b"s", b"plain")
    return lib


class DefaultPool:
    """The current device's default stream-ordered memory pool, read through
    the driver API (the library's scratch comes from this pool)."""

    def __init__(self):
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuCtxGetDevice(ctypes.byref(dev)) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def get(self, attr):
        v = ctypes.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return v.value

    def reset_high(self):
        zero = ctypes.c_uint64(0)  # resets the high watermark to the current use
        assert self.cu.cuMemPoolSetAttribute(self.pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                             ctypes.byref(zero)) == 0


def _device_matrix(torch, lib, rows, cols, seed, matrix_id):
    """rows x cols column-major FP32 device matrix (torch stores it transposed)."""
    t = torch.empty(cols, rows, dtype=torch.float32, device="cuda")
    assert lib.mublis_b200_fill_s(ctypes.c_void_p(t.data_ptr()), rows, cols, rows, seed,
                                  matrix_id, 0) == 0
    return t


def _normwise(got, ref, a, b, c0, alpha, beta):
    den = abs(alpha) * np.linalg.norm(a) * np.linalg.norm(b) + abs(beta) * np.linalg.norm(c0)
    return np.linalg.norm(got.astype(np.float64) - ref.astype(np.float64)) / den


def _compare_with_sgemm(torch, lib, m, n, k, ta, tb, seed, alpha=0.75, beta=0.25):
    """Runs mublis_sgemm and the allocation-free entry point on the same
    device operands; checks that the latter takes no memory and returns the
    normwise difference."""
    a = _device_matrix(torch, lib, k if ta else m, m if ta else k, seed, 0)
    b = _device_matrix(torch, lib, n if tb else k, k if tb else n, seed, 1)
    c0 = _device_matrix(torch, lib, m, n, seed, 2)
    c_ref, c_new = c0.clone(), c0.clone()
    lda, ldb = (k if ta else m), (n if tb else k)
    torch.cuda.synchronize()
    st = lib.mublis_sgemm(ta, tb, m, n, k, alpha, a.data_ptr(), 1, lda, b.data_ptr(), 1, ldb,
                          beta, c_ref.data_ptr(), 1, m)
    assert st == 0, mb.last_error(lib)
    torch.cuda.synchronize()
    pool = DefaultPool()
    used_before = pool.get(CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
    pool.reset_high()
    free_before = torch.cuda.mem_get_info()[0]
    st = lib.mublis_b200_sgemm_noalloc(ta, tb, m, n, k, alpha, a.data_ptr(), 1, lda,
                                       b.data_ptr(), 1, ldb, beta, c_new.data_ptr(), 1, m)
    assert st == 0, mb.last_error(lib)
    torch.cuda.synchronize()
    assert pool.get(CU_MEMPOOL_ATTR_USED_MEM_HIGH) == used_before, "the call took pool memory"
    assert torch.cuda.mem_get_info()[0] == free_before
    ref = c_ref.cpu().numpy().T
    got = c_new.cpu().numpy().T
    assert np.isfinite(got).all()
    return _normwise(got, ref, a.cpu().numpy(), b.cpu().numpy(), c0.cpu().numpy(), alpha, beta)


def test_noalloc_matches_sgemm_on_two_calls_in_a_row(lib):
    torch = pytest.importorskip("torch")
    for i, (m, n, k, ta, tb, seed) in enumerate([(700, 513, 300, 0, 0, 11),
                                                 (1024, 1000, 1024, 1, 1, 12)]):
        err = _compare_with_sgemm(torch, lib, m, n, k, ta, tb, seed)
        assert err <= 4 * k * 2.0 ** -24, (i, err)


def test_noalloc_at_the_exact_limit(lib):
    """(2048 + 2048) * 2048 floats is exactly the scratch size: the B panel
    ends on the array's last element."""
    torch = pytest.importorskip("torch")
    err = _compare_with_sgemm(torch, lib, 2048, 2048, 2048, 0, 1, 13)
    assert err <= 4 * 2048 * 2.0 ** -24, err


@pytest.mark.parametrize("mnk", [(2048, 2048, 2049), (4096, 4096, 4096)],
                         ids=["one-k-block-over", "far-over"])
def test_noalloc_refuses_sizes_beyond_the_scratch_limit(lib, mnk):
    torch = pytest.importorskip("torch")
    m, n, k = mnk
    a = _device_matrix(torch, lib, m, k, 3, 0)
    b = _device_matrix(torch, lib, k, n, 3, 1)
    c = _device_matrix(torch, lib, m, n, 3, 2)
    keep = c.clone()
    torch.cuda.synchronize()
    st = lib.mublis_b200_sgemm_noalloc(0, 0, m, n, k, 1.0, a.data_ptr(), 1, m, b.data_ptr(), 1, k,
                                       0.5, c.data_ptr(), 1, m)
    assert st != 0
    assert "maximum" in mb.last_error(lib)
    torch.cuda.synchronize()
    assert torch.equal(c, keep)


def test_noalloc_empty_sizes_return_first(lib):
    """An empty output returns 0 before the other sizes are checked, as
    mublis_sgemm does."""
    for m, n, k in ((0, -1, 5), (-1, 0, 5), (0, 3, -2)):
        assert lib.mublis_sgemm(0, 0, m, n, k, 1.0, None, 1, 1, None, 1, 1, 0.0, None, 1,
                                1) == 0
        assert lib.mublis_b200_sgemm_noalloc(0, 0, m, n, k, 1.0, None, 1, 1, None, 1, 1, 0.0,
                                             None, 1, 1) == 0
    assert lib.mublis_b200_sgemm_noalloc(0, 0, -1, 3, 2, 1.0, None, 1, 1, None, 1, 1, 0.0,
                                         None, 1, 1) != 0
