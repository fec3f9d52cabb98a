"""Generate tests/golden/l3_golden.npz from the reference's own build.

Run from the repository root after `make -C oracle` (which compiles the
reference's C sources into oracle/_ref/):

    python tests/golden/make_golden.py

For every case in CASES the inputs are the seeded Philox draws of
tests/cases.py (regenerated at test time from the seed, so only outputs are
stored); the stored output is what the reference's `linux_avx2` build
(oracle/_ref/avx2/libmublis.so) returns through its cblas_* entry points.
The case list covers every routine in both precisions and both layouts,
every side/uplo/trans/diag flag, ragged and tiny sizes, m/n/k = 0 and 1,
alpha = 0 and beta = 0.
"""
from __future__ import annotations

import itertools
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as orc  # noqa: E402
from tests import cases as cs  # noqa: E402

OUT = Path(__file__).resolve().parent / "l3_golden.npz"


def golden_cases():
    out = []
    seed = 11
    sizes = [(1, 1, 1), (7, 5, 3), (19, 13, 11), (33, 24, 9)]
    for dt, order in itertools.product(("float32", "float64"), ("F", "C")):
        for (m, n, k) in sizes:
            seed += 1
            base = dict(dtype=dt, order=order, seed=seed)
            for ta, tb in ((False, False), (True, False), (False, True), (True, True)):
                out.append(dict(base, routine="gemm", m=m, n=n, k=k, ta=ta, tb=tb, alpha=0.75,
                                beta=0.25))
            for right, lower in itertools.product((False, True), repeat=2):
                out.append(dict(base, routine="symm", m=m, n=n, k=0, right=right, lower=lower,
                                alpha=0.75, beta=0.25))
            for r in ("syrk", "syr2k"):
                for ta, lower in itertools.product((False, True), repeat=2):
                    out.append(dict(base, routine=r, m=n, n=n, k=k, ta=ta, lower=lower,
                                    alpha=0.75, beta=0.25))
            for r in ("trmm", "trsm"):
                for right, lower, ta, unit in itertools.product((False, True), repeat=4):
                    if (m, n, k) == (33, 24, 9) and (ta or unit):
                        continue
                    out.append(dict(base, routine=r, m=m, n=n, k=0, right=right, lower=lower,
                                    ta=ta, unit=unit, alpha=0.75))
    # Edge semantics: alpha == 0 (beta-scale only, A/B never read), beta == 0
    # (C never read), empty k, empty m/n.
    for dt in ("float32", "float64"):
        base = dict(dtype=dt, order="F", seed=99)
        out.append(dict(base, routine="gemm", m=9, n=6, k=4, ta=False, tb=False, alpha=0.0,
                        beta=0.5))
        out.append(dict(base, routine="gemm", m=9, n=6, k=4, ta=False, tb=True, alpha=1.5,
                        beta=0.0))
        out.append(dict(base, routine="gemm", m=9, n=6, k=0, ta=False, tb=False, alpha=1.5,
                        beta=0.5))
        out.append(dict(base, routine="gemm", m=0, n=6, k=4, ta=False, tb=False, alpha=1.5,
                        beta=0.5))
        out.append(dict(base, routine="syrk", m=8, n=8, k=5, ta=False, lower=True, alpha=0.0,
                        beta=0.0))
        out.append(dict(base, routine="trmm", m=8, n=5, k=0, right=False, lower=True, ta=False,
                        unit=False, alpha=0.0))
        out.append(dict(base, routine="trsm", m=8, n=5, k=0, right=True, lower=False, ta=True,
                        unit=True, alpha=0.0))
    return out


def main():
    ref = orc.reference("avx2")
    cases = golden_cases()
    arrays = {}
    for i, c in enumerate(cases):
        a, b, c0 = cs.build(c)
        out = c0.copy(order="K")
        cs.cblas_call(ref, c, a, b, out)
        arrays[f"out{i}"] = out
    np.savez_compressed(OUT, cases=np.array(json.dumps(cases)), **arrays)
    print(f"wrote {len(cases)} cases to {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
