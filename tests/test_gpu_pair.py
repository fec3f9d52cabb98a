"""The tensor-core forms on CTA pairs (cta_group::2) give the bits of the
same forms on one SM per tile (GPU).

MUBLIS_B200_TC_PAIR is read once per process, so each variant runs in a
child process on the same seeded device operands: the FP32 forms (fp16x3,
bf16x3, bf16x6) at sizes from one pair tile to ragged multi-tile shapes, and
the modular Ozaki form in both precisions (pairs are taken below 576 tiles,
so every size here runs on pairs when allowed).  Each result is also held
to its form's normwise bound against an FP64 product.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[2])
import mublis_b200 as mb
lib = mb.load()
assert lib.mublis_b200_init() == 0
out = {}
g = torch.Generator(device="cuda").manual_seed(5)
cases = [("s", f, n, k) for f in ("fp16x3", "bf16x3", "bf16x6") for n, k in ((256, 64), (600, 300), (1030, 700))]
cases += [(p, "ozaki2", n, k) for p in ("s", "d") for n, k in ((256, 100), (700, 1300))]
for p, form, n, k in cases:
    dt = torch.float32 if p == "s" else torch.float64
    A = torch.rand(n, k, device="cuda", generator=g, dtype=dt) * 2 - 1
    B = torch.rand(k, n, device="cuda", generator=g, dtype=dt) * 2 - 1
    C0 = torch.rand(n, n, device="cuda", generator=g, dtype=dt) * 2 - 1
    a, b, c = A.T.contiguous(), B.T.contiguous(), C0.T.contiguous()
    torch.cuda.synchronize()
    assert lib.mublis_b200_set_form(p.encode(), form.encode()) == 0
    fn = getattr(lib, f"mublis_{p}gemm")
    assert fn(0, 0, n, n, k, 0.75, a.data_ptr(), 1, n, b.data_ptr(), 1, k, 0.25,
              c.data_ptr(), 1, n) == 0, mb.last_error(lib)
    torch.cuda.synchronize()
    lib.mublis_b200_set_form(p.encode(), b"plain")
    ref = 0.75 * (A.double() @ B.double()) + 0.25 * C0.double()
    den = 0.75 * A.double().norm() * B.double().norm() + 0.25 * C0.double().norm()
    key = f"{p}_{form}_{n}_{k}"
    out[key] = c.cpu().numpy()
    out[key + "_err"] = np.array(float((c.T.double() - ref).norm() / den))
np.savez(sys.argv[1], **out)
"""


def run_child(path, pair):
    env = dict(os.environ)
    env["MUBLIS_B200_TC_PAIR"] = "1" if pair else "0"
    subprocess.run([sys.executable, "-c", CHILD, str(path), ROOT], env=env, check=True,
                   timeout=600)
    return np.load(path)


def test_pair_kernels_equal_single_sm_kernels(tmp_path):
    pytest.importorskip("torch")
    on = run_child(tmp_path / "pair.npz", True)
    off = run_child(tmp_path / "single.npz", False)
    keys = [k for k in on.files if not k.endswith("_err")]
    assert keys
    for key in keys:
        np.testing.assert_array_equal(on[key].view(np.uint8), off[key].view(np.uint8), err_msg=key)
        p, form, n, k = key.split("_")
        u = 2.0 ** -24 if p == "s" else 2.0 ** -53
        # fp16x3 / bf16x6 / ozaki2 within plain's 4 k u; bf16x3 keeps 16 of
        # the 24 input bits (2^-19 normwise, as tests/test_gpu_forms.py holds it).
        bound = 2.0 ** -19 if form == "bf16x3" else 4 * int(k) * u
        assert float(on[key + "_err"]) <= bound, (key, float(on[key + "_err"]))
