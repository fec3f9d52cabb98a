"""The bounded device waits, exercised without a fault or a hang.

Every mbarrier wait in the library's warp-specialised kernels is bounded
(%globaltimer); when one runs out the CTA raises its abort flag and the
mapped error word, the kernel returns, and the host call reports status 4.
mublis_b200_test_stall_next arms this path for one launch of the FP64
tensor-pipe GEMM: that launch's producer issues no loads (a flag that
nothing sets, from the consumers' side) and its waits are bounded by a
short limit, so the consumers' first wait runs out after the limit.

Checked: the stalled call returns 4 with a "timed out" message and leaves C
unchanged (no tile reached its epilogue); the very next call on the same
context succeeds and matches the oracle; the stall is one-shot; limits
outside (0, 2 s] are refused.
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
    lib.mublis_b200_set_form(b"d", b"plain")
    return lib


def _dgemm(lib, a, b, c, m, n, k):
    return lib.mublis_dgemm(0, 0, m, n, k, 0.75, a.ctypes.data, 1, m, b.ctypes.data, 1, k, 0.25,
                            c.ctypes.data, 1, m)


def test_stalled_launch_times_out_and_the_context_stays_usable(lib):
    m, n, k = 384, 320, 256
    a = orc.fill(m, k, np.float64, 31, 0)
    b = orc.fill(k, n, np.float64, 31, 1)
    c0 = orc.fill(m, n, np.float64, 31, 2)

    assert lib.mublis_b200_test_stall_next(1_000_000) == 0  # 1 ms
    c = c0.copy(order="F")
    st = _dgemm(lib, a, b, c, m, n, k)
    assert st == 4, (st, mb.last_error(lib))
    assert "timed out" in mb.last_error(lib)
    np.testing.assert_array_equal(c, c0)

    # The next call (stall consumed) runs normally on the same context.
    c = c0.copy(order="F")
    assert _dgemm(lib, a, b, c, m, n, k) == 0, mb.last_error(lib)
    case = dict(routine="gemm", dtype="float64", order="F", m=m, n=n, k=k, ta=False, tb=False,
                alpha=0.75, beta=0.25, seed=31)
    ref = c0.copy(order="F")
    cs.oracle_call(case, a, b, ref)
    assert cs.normwise_error(case, c, ref, a, b, c0) <= 4 * k * 2.0 ** -53

    # And again: one-shot.
    c2 = c0.copy(order="F")
    assert _dgemm(lib, a, b, c2, m, n, k) == 0
    np.testing.assert_array_equal(c2, c)


def test_stall_limits_are_checked(lib):
    assert lib.mublis_b200_test_stall_next(0) != 0
    assert lib.mublis_b200_test_stall_next(3_000_000_000) != 0
