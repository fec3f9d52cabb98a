"""Pins the oracle before anything is checked against it (CPU only).

* Philox4x32-10 against the Random123 known-answer vectors;
* the C restatement (oracle/mublis_oracle.c) against
  - the reference's own builds (oracle/_ref, configs `reference` and `avx2`)
    on the reference test-suite's full case matrix (check_cblas.py:224-473),
  - scipy.linalg.blas, the reference test-suite's own oracle, on the same
    cases and with its tolerances,
  - the committed golden outputs of the reference build
    (tests/golden/l3_golden.npz, made by tests/golden/make_golden.py);
* the generic driver's domain/structure semantics against the reference's
  mublis_l3_{s,d}driver for combinations whose result does not depend on
  the reference's block sizes.
"""
import ctypes
import json
from pathlib import Path

import numpy as np
import pytest

import mublis_b200 as mb
from oracle import oracle as orc
from tests import cases as cs

GOLDEN = Path(__file__).resolve().parent / "golden" / "l3_golden.npz"

REF_MATRIX = cs.reference_matrix()


def test_philox_known_answers():
    # Random123 kat_vectors for philox4x32_10.
    assert orc.philox_ctr([0, 0, 0, 0], [0, 0]) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert orc.philox_ctr([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == (
        0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert orc.philox_ctr([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                          [0xA4093822, 0x299F31D0]) == (0xD16CFE09, 0x94FDCCEB, 0x5001E420,
                                                        0x24126EA1)


def test_draws_ranges():
    u = orc.fill(300, 200, np.float64, 0, 0)
    assert u.min() >= -1 and u.max() < 1 and abs(u.mean()) < 0.01
    w = orc.fill(300, 200, np.float32, 0, 0, orc.WIDE)
    aw = np.abs(w)
    assert aw.min() >= 2.0 ** -10 and aw.max() < 2.0 ** 11
    d = orc.fill(50, 50, np.float32, 3, 1, orc.DIAG)
    assert d.min() >= 1 and d.max() < 2
    # column-major counter: element (i, j) uses index i + j*m
    x = orc.fill(7, 3, np.float32, 5, 2)
    w0 = orc.philox(1 + 2 * 7, 5, 2)[0]
    assert x[1, 2] == np.float32((w0 >> 8) * 2.0 ** -23 - 1)


def _run(case, runner):
    a, b, c0 = cs.build(case)
    out = c0.copy(order="K")
    runner(case, a, b, out)
    return a, b, c0, out


@pytest.mark.parametrize("case", REF_MATRIX, ids=[cs.case_id(c) for c in REF_MATRIX])
@pytest.mark.parametrize("config", ["reference", "avx2"])
def test_restatement_matches_reference_build(case, config):
    path = orc.ref_lib_path(config)
    if not path.is_file():
        pytest.skip("reference build not present")
    ref = orc.reference(config)
    a, b, c0, mine = _run(case, cs.oracle_call)
    _, _, _, theirs = _run(case, lambda c, x, y, z: cs.cblas_call(ref, c, x, y, z))
    rtol, atol = cs.REF_TOL[np.dtype(case["dtype"])]
    mask = cs.active_mask(case)
    np.testing.assert_allclose(mine[mask], theirs[mask], rtol=rtol, atol=atol)
    # untouched triangle bit-identical (check_cblas.py:355-363)
    np.testing.assert_array_equal(mine[~mask], c0[~mask])


@pytest.mark.parametrize("case", REF_MATRIX, ids=[cs.case_id(c) for c in REF_MATRIX])
def test_restatement_matches_scipy(case):
    a, b, c0, mine = _run(case, cs.oracle_call)
    expected = cs.scipy_expected(case, a, b, c0)
    rtol, atol = cs.REF_TOL[np.dtype(case["dtype"])]
    mask = cs.active_mask(case)
    np.testing.assert_allclose(mine[mask], np.asarray(expected)[mask], rtol=rtol, atol=atol)


def _golden():
    data = np.load(GOLDEN)
    cases = json.loads(str(data["cases"]))
    return cases, data


GOLDEN_CASES, _ = _golden()


@pytest.mark.parametrize("idx", range(len(GOLDEN_CASES)),
                         ids=[cs.case_id(c) for c in GOLDEN_CASES])
def test_restatement_matches_golden(idx):
    cases, data = _golden()
    case = cases[idx]
    expected = data[f"out{idx}"]
    a, b, c0, mine = _run(case, cs.oracle_call)
    dt = np.dtype(case["dtype"])
    mask = cs.active_mask(case)
    if mine.size == 0:
        return
    err = cs.normwise_error(case, mine, expected, a, b, c0)
    tol = 4 * max(cs.inner_dim(case), 1) * cs.EPS[dt]
    assert err <= tol, (err, tol)
    np.testing.assert_array_equal(mine[~mask], expected[~mask])
    assert np.isfinite(mine[mask]).all()


# Generic-driver products whose result is independent of block sizes: the
# domain relations agree with the operands' triangular structure.
DRIVER_CASES = [
    # triangular (lower) x general with pi = LOWER  (TRMM-like)
    dict(jp=0, ji=0, pi=1, a=(2, 1, 0), b=(0, 0, 0)),
    # general x triangular (upper) with jp = UPPER
    dict(jp=2, ji=0, pi=0, a=(0, 0, 0), b=(2, 2, 0)),
    # lower-triangular x lower-triangular, unit diagonals, lower output
    dict(jp=1, ji=1, pi=1, a=(2, 1, 1), b=(2, 1, 1)),
    # symmetric (upper stored) x general, upper output
    dict(jp=0, ji=2, pi=0, a=(1, 2, 0), b=(0, 0, 0)),
    # general x symmetric (lower stored)
    dict(jp=0, ji=0, pi=0, a=(0, 0, 0), b=(1, 1, 0)),
]


@pytest.mark.parametrize("dc", DRIVER_CASES)
@pytest.mark.parametrize("p", ["s", "d"])
def test_restated_driver_matches_reference_driver(dc, p):
    if not orc.ref_lib_path("avx2").is_file():
        pytest.skip("reference build not present")
    dt = np.float32 if p == "s" else np.float64
    m = n = k = 37
    a = orc.fill(m, k, dt, 3, 0)
    b = orc.fill(k, n, dt, 3, 1)
    c0 = orc.fill(m, n, dt, 3, 2)
    # poison what structured operands must not read
    for x, (struc, uplo, diag) in ((a, dc["a"]), (b, dc["b"])):
        if struc in (1, 2):
            tri = np.triu_indices(37, 1) if uplo == 1 else np.tril_indices(37, -1)
            x[tri] = np.nan
        if struc == 2 and diag == 1:
            np.fill_diagonal(x, np.nan)
    prod = mb.Product(mb.Domain(dc["jp"], dc["ji"], dc["pi"]), mb.Operand(*dc["a"]),
                      mb.Operand(*dc["b"]))
    outs = []
    for fn in (getattr(orc.restated(), f"oracle_l3_{p}driver"),
               getattr(orc.reference("avx2"), f"mublis_l3_{p}driver")):
        c = c0.copy(order="F")
        st = fn(m, n, k, 0.75, a.ctypes.data, 1, m, b.ctypes.data, 1, k, 0.25, c.ctypes.data, 1,
                m, ctypes.byref(prod))
        assert st == 0
        outs.append(c)
    tol = 4 * k * (2.0 ** -24 if p == "s" else 2.0 ** -53)
    fa = np.linalg.norm(np.nan_to_num(a)) * np.linalg.norm(np.nan_to_num(b)) * 0.75
    err = np.linalg.norm(np.nan_to_num(outs[0] - outs[1])) / (fa + 0.25 * np.linalg.norm(c0))
    assert np.isfinite(outs[0]).all() and np.isfinite(outs[1]).all()
    assert err <= tol


@pytest.mark.parametrize("n,panel", [(300, 64), (257, 100)])
def test_parallel_reference_family_panels_match_whole_calls(n, panel):
    """The benchmark's reference arm cuts every call of the family into
    column panels issued as separate reference calls (SYRK/SYR2K: a
    diagonal-block SYRK/SYR2K plus GEMMs below it) to use every host thread.
    Its check mode recomputes each call whole on the same inputs: the panels
    must give the same result up to rounding (a wrong cut would differ by
    O(1))."""
    import json
    import subprocess
    lib = orc.ref_lib_path("avx2")
    if not lib.is_file() or not orc.REF_BENCH.is_file():
        pytest.skip("reference build not present")
    out = subprocess.run([str(orc.REF_BENCH), str(lib), "family_par", "x", str(n), str(n),
                          str(n), "4", "1", "0", str(-panel)], check=True, capture_output=True,
                         text=True).stdout
    r = json.loads(out.strip().splitlines()[-1])
    assert r["routine"] == "family_par_check"
    assert r["tasks"] == 18 * -(-n // panel)
    assert r["max_rel_diff"] <= 1e-5, r
