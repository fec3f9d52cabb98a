"""Host-pointer calls large enough to be moved through the device in column
panels (host copy-in, arithmetic and copy-out of neighbouring panels
overlapped on three streams).

Every case is run twice through cblas_*: once on host numpy arrays (the
pipelined or triangle-staged path) and once on device copies of the same
bytes (one call, no staging).  With the plain forms each output element is summed in the same
order whatever the panel width, so the two results must be bit-identical
(the device path itself is checked against the oracle by the parity
suite).
"""
import types

import numpy as np
import pytest

import mublis_b200 as mb
from tests import cases as cs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    lib = mb.load()
    assert lib.mublis_b200_init() == 0, mb.last_error(lib)
    for p in (b"s", b"d"):
        lib.mublis_b200_set_form(p, b"plain")
    return lib


class DeviceCopy:
    """The bytes of a numpy array in device memory, with the array's shape
    and strides, usable wherever tests/cases.py takes an array."""

    def __init__(self, torch, x):
        flat = np.frombuffer(x.tobytes(order="A"), dtype=x.dtype)
        self.buf = torch.from_numpy(flat.copy()).cuda()
        self.shape, self.strides, self.itemsize, self.size = x.shape, x.strides, x.itemsize, x.size
        self.dtype = x.dtype
        self.order = "F" if x.flags["F_CONTIGUOUS"] and not x.flags["C_CONTIGUOUS"] else "C"
        self.ctypes = types.SimpleNamespace(data=self.buf.data_ptr())

    def host(self):
        flat = self.buf.cpu().numpy()
        return np.ndarray(self.shape, dtype=self.dtype, buffer=flat.tobytes(), order=self.order)


CASES = [
    dict(routine="gemm", dtype="float32", order="F", m=1536, n=4096, k=1024, ta=False, tb=False,
         alpha=0.75, beta=0.25, seed=31),
    dict(routine="gemm", dtype="float64", order="F", m=1024, n=3072, k=1024, ta=True, tb=True,
         alpha=0.75, beta=0.25, seed=32),
    dict(routine="gemm", dtype="float32", order="C", m=2048, n=4096, k=512, ta=False, tb=True,
         alpha=1.0, beta=0.0, seed=33),
    dict(routine="symm", dtype="float64", order="F", m=1024, n=4096, right=False, lower=True,
         alpha=0.75, beta=0.25, seed=34),
    dict(routine="trmm", dtype="float64", order="F", m=1024, n=4096, right=False, lower=True,
         ta=False, unit=False, alpha=0.75, seed=35),
    dict(routine="trsm", dtype="float32", order="F", m=2048, n=4096, right=False, lower=True,
         ta=False, unit=False, alpha=0.75, seed=36),
    dict(routine="trsm", dtype="float64", order="F", m=4096, n=1024, right=True, lower=False,
         ta=True, unit=True, alpha=0.5, seed=37),
    # lower-triangle outputs: C moves in triangle panels (copied in even for
    # beta == 0, since the diagonal blocks carry upper elements)
    dict(routine="syrk", dtype="float64", order="F", m=4096, n=4096, k=1024, ta=False,
         lower=True, alpha=0.75, beta=0.25, seed=38),
    dict(routine="syrk", dtype="float32", order="F", m=4096, n=4096, k=768, ta=True,
         lower=True, alpha=1.0, beta=0.0, seed=39),
    dict(routine="syr2k", dtype="float32", order="F", m=4096, n=4096, k=1536, ta=False,
         lower=True, alpha=0.75, beta=0.25, seed=40),
    # row-major lower is a column-major upper triangle: staged as a triangle,
    # not pipelined
    dict(routine="syr2k", dtype="float64", order="C", m=3072, n=3072, k=512, ta=True,
         lower=True, alpha=0.5, beta=0.5, seed=41),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c['routine']}-{c['dtype']}-{c['order']}")
def test_pipelined_host_call_matches_device_call(lib, case):
    torch = pytest.importorskip("torch")
    if case["routine"] in ("gemm", "symm"):
        case.setdefault("k", case["m"])
    elif case["routine"] in ("trmm", "trsm"):
        case.setdefault("k", case["m"] if not case["right"] else case["n"])
    a, b, c0 = cs.build(case)
    host_out = c0.copy(order="K")
    cs.cblas_call(lib, case, a, b, host_out)
    da, dc = DeviceCopy(torch, a), DeviceCopy(torch, c0)
    db = None if b is None else DeviceCopy(torch, b)
    torch.cuda.synchronize()
    cs.cblas_call(lib, case, da, db, dc)
    torch.cuda.synchronize()
    dev_out = dc.host()
    assert np.isfinite(host_out).all()
    np.testing.assert_array_equal(host_out, dev_out)
