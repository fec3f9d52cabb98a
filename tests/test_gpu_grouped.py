"""Grouped launches: many independent GEMMs / TRSMs of
uneven sizes in one persistent launch, and plans (autotuned tiles + CUDA
graph replay).

Each grouped result is compared with the library's single-call path on the
same device operands (normwise relative error <= 4 * k * u, the suite's
tolerance) and, for a few problems, with the oracle restatement.
"""
import ctypes

import numpy as np
import pytest

import mublis_b200 as mb
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


GemmProblem, TrsmProblem = mb.GemmProblem, mb.TrsmProblem


@pytest.fixture(scope="module")
def glib():
    lib = mb.load()
    assert lib.mublis_b200_init() == 0, mb.last_error(lib)
    for p in (b"s", b"d"):
        lib.mublis_b200_set_form(p, b"plain")
    return lib


def log_uniform_int(rng, lo, hi, size):
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size))).astype(int)


def make_gemm_set(torch, p, count, seed, lo=16, hi=512):
    dt = torch.float32 if p == "s" else torch.float64
    rng = np.random.default_rng(seed)
    mnk = log_uniform_int(rng, lo, hi, (count, 3))
    probs, keep = [], []
    for q in range(count):
        m, n, k = (int(x) for x in mnk[q])
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        a = torch.rand((m, k) if ta else (k, m), dtype=dt, device="cuda") * 2 - 1
        b = torch.rand((k, n) if tb else (n, k), dtype=dt, device="cuda") * 2 - 1
        c = torch.rand((n, m), dtype=dt, device="cuda") * 2 - 1
        al, be = rng.uniform(0.5, 1.5, 2)
        # torch tensors are row-major: a (rows, cols) row-major buffer is the
        # column-major transpose, so lda is the row length.
        probs.append(GemmProblem(ta, tb, m, n, k, al, be, a.data_ptr(), a.shape[1], b.data_ptr(),
                                 b.shape[1], c.data_ptr(), m))
        keep.append((a, b, c))
    return probs, keep


def single_call(lib, p, pr):
    fn = getattr(lib, f"mublis_{p}gemm")
    return fn(pr.trans_a, pr.trans_b, pr.m, pr.n, pr.k, pr.alpha, pr.a, 1, pr.lda, pr.b, 1,
              pr.ldb, pr.beta, pr.c, 1, pr.ldc)


@pytest.mark.parametrize("p", ["s", "d"])
def test_grouped_gemm_matches_single_calls(glib, p):
    torch = pytest.importorskip("torch")
    probs, keep = make_gemm_set(torch, p, 96, seed=1)
    c0 = [c.clone() for _, _, c in keep]
    arr = (GemmProblem * len(probs))(*probs)
    assert glib.mublis_b200_gemm_grouped(p.encode(), arr, len(probs)) == 0, mb.last_error(glib)
    grouped = [c.clone() for _, _, c in keep]
    u = 2.0 ** -24 if p == "s" else 2.0 ** -53
    for q, pr in enumerate(probs):
        keep[q][2].copy_(c0[q])
        assert single_call(glib, p, pr) == 0
        a, b, _ = keep[q]
        den = abs(pr.alpha) * a.norm().item() * b.norm().item() + abs(pr.beta) * c0[q].norm().item()
        err = (grouped[q].double() - keep[q][2].double()).norm().item() / den
        assert err <= 4 * pr.k * u, (q, pr.m, pr.n, pr.k, err)


def test_grouped_gemm_against_oracle(glib):
    torch = pytest.importorskip("torch")
    m, n, k = 37, 129, 200
    a = orc.fill(m, k, np.float32, 5, 0)
    b = orc.fill(k, n, np.float32, 5, 1)
    c0 = orc.fill(m, n, np.float32, 5, 2)
    ta, tb, tc = (torch.from_numpy(x.T.copy()).cuda() for x in (a, b, c0))
    pr = GemmProblem(0, 0, m, n, k, 0.75, 0.25, ta.data_ptr(), m, tb.data_ptr(), k,
                     tc.data_ptr(), m)
    assert glib.mublis_b200_gemm_grouped(b"s", (GemmProblem * 1)(pr), 1) == 0
    ref = c0.copy(order="F")
    assert orc.restated().oracle_sgemm(0, 0, m, n, k, 0.75, a.ctypes.data, 1, m, b.ctypes.data,
                                       1, k, 0.25, ref.ctypes.data, 1, m) == 0
    got = tc.cpu().numpy().T
    err = np.linalg.norm(got - ref) / (0.75 * np.linalg.norm(a) * np.linalg.norm(b) +
                                       0.25 * np.linalg.norm(c0))
    assert err <= 4 * k * 2.0 ** -24


@pytest.mark.parametrize("p", ["s", "d"])
def test_plan_replay_equals_grouped_call(glib, p):
    torch = pytest.importorskip("torch")
    probs, keep = make_gemm_set(torch, p, 64, seed=3)
    c0 = [c.clone() for _, _, c in keep]
    arr = (GemmProblem * len(probs))(*probs)
    plan = ctypes.c_void_p()
    assert glib.mublis_b200_plan_gemm_grouped(p.encode(), arr, len(probs), ctypes.byref(plan)) == 0
    # planning (autotuning trials included) leaves C as it was
    for q in range(len(probs)):
        assert torch.equal(keep[q][2], c0[q])
    assert glib.mublis_b200_plan_run(plan) == 0
    replay = [c.clone() for _, _, c in keep]
    for q in range(len(probs)):
        keep[q][2].copy_(c0[q])
    assert glib.mublis_b200_gemm_grouped(p.encode(), arr, len(probs)) == 0
    for q in range(len(probs)):
        assert torch.equal(replay[q], keep[q][2])  # same tiles -> bit-identical
    assert glib.mublis_b200_plan_destroy(plan) == 0


def make_trsm_set(torch, p, count, seed):
    dt = torch.float32 if p == "s" else torch.float64
    rng = np.random.default_rng(seed)
    orders = log_uniform_int(rng, 32, 256, count)
    nrhs = log_uniform_int(rng, 1, 128, count)
    probs, keep = [], []
    for q in range(count):
        m, n = int(orders[q]), int(nrhs[q])
        a = (torch.rand(m, m, dtype=dt, device="cuda") * 2 - 1) / m
        a.diagonal().copy_(torch.rand(m, dtype=dt, device="cuda") + 1)
        b = torch.rand(n, m, dtype=dt, device="cuda") * 2 - 1
        uplo = mb.M_LOWER if q % 2 == 0 else mb.M_UPPER
        trans = q % 3 == 0
        diag = mb.M_UNIT if q % 5 == 0 else mb.M_NON_UNIT
        probs.append(TrsmProblem(uplo, int(trans), diag, m, n, float(rng.uniform(0.5, 1.5)),
                                 a.data_ptr(), m, b.data_ptr(), m))
        keep.append((a, b))
    return probs, keep


@pytest.mark.parametrize("p", ["s", "d"])
def test_grouped_trsm_matches_single_calls(glib, p):
    torch = pytest.importorskip("torch")
    probs, keep = make_trsm_set(torch, p, 48, seed=4)
    b0 = [b.clone() for _, b in keep]
    arr = (TrsmProblem * len(probs))(*probs)
    assert glib.mublis_b200_trsm_grouped(p.encode(), arr, len(probs)) == 0, mb.last_error(glib)
    grouped = [b.clone() for _, b in keep]
    u = 2.0 ** -24 if p == "s" else 2.0 ** -53
    fn = getattr(glib, f"mublis_{p}trsm")
    for q, pr in enumerate(probs):
        keep[q][1].copy_(b0[q])
        assert fn(mb.M_LEFT, pr.uplo, pr.trans_a, pr.diag, pr.m, pr.n, pr.alpha, pr.a, 1, pr.lda,
                  pr.b, 1, pr.ldb) == 0
        ref = keep[q][1].double()
        err = (grouped[q].double() - ref).norm().item() / ref.norm().item()
        assert err <= 4 * pr.m * u, (q, pr.m, pr.n, err)


@pytest.mark.parametrize("p", ["s", "d"])
def test_trsm_plan_replay(glib, p):
    torch = pytest.importorskip("torch")
    probs, keep = make_trsm_set(torch, p, 32, seed=6)
    b0 = [b.clone() for _, b in keep]
    arr = (TrsmProblem * len(probs))(*probs)
    plan = ctypes.c_void_p()
    assert glib.mublis_b200_plan_trsm_grouped(p.encode(), arr, len(probs), ctypes.byref(plan)) == 0
    assert glib.mublis_b200_plan_run(plan) == 0
    replay = [b.clone() for _, b in keep]
    for q in range(len(probs)):
        keep[q][1].copy_(b0[q])
    assert glib.mublis_b200_trsm_grouped(p.encode(), arr, len(probs)) == 0
    for q in range(len(probs)):
        assert torch.equal(replay[q], keep[q][1])
    assert glib.mublis_b200_plan_destroy(plan) == 0


def test_tuned_table_round_trip(glib, tmp_path):
    """The autotuner's choices survive a save / reset / load cycle: a plan
    created after loading the table launches no tuning trials; a table keyed
    to another GPU loads nothing."""
    torch = pytest.importorskip("torch")
    probs, keep = make_gemm_set(torch, "s", 40, seed=9)
    arr = (GemmProblem * len(probs))(*probs)
    assert glib.mublis_b200_tune_reset() == 0

    def plan_launches():
        plan = ctypes.c_void_p()
        n0 = glib.mublis_b200_launch_count()
        assert glib.mublis_b200_plan_gemm_grouped(b"s", arr, len(probs), ctypes.byref(plan)) == 0
        n1 = glib.mublis_b200_launch_count()
        assert glib.mublis_b200_plan_destroy(plan) == 0
        return n1 - n0

    untuned = plan_launches()
    path = tmp_path / "tune.txt"
    assert glib.mublis_b200_tune_save(str(path).encode()) == 0, mb.last_error(glib)
    lines = path.read_text().splitlines()
    assert lines[0].startswith("mublis_b200-tune ") and "driver=" in lines[0]
    choices = [ln for ln in lines[1:] if ln.startswith("gemm ")]
    assert choices

    assert glib.mublis_b200_tune_reset() == 0
    entries = ctypes.c_int(-1)
    assert glib.mublis_b200_tune_load(str(path).encode(), ctypes.byref(entries)) == 0
    assert entries.value == len(choices)
    assert plan_launches() < untuned  # no trial launches once the table is loaded

    other = tmp_path / "other.txt"
    other.write_text("mublis_b200-tune Another_GPU sms=1 cc=1.0 driver=1 table=1\ngemm 0 0 0 1\n")
    assert glib.mublis_b200_tune_reset() == 0
    assert glib.mublis_b200_tune_load(str(other).encode(), ctypes.byref(entries)) == 0
    assert entries.value == 0
    missing = tmp_path / "missing.txt"
    assert glib.mublis_b200_tune_load(str(missing).encode(), ctypes.byref(entries)) == 0
    assert entries.value == 0


@pytest.fixture
def fp16x3(glib):
    glib.mublis_b200_set_form(b"s", b"fp16x3")
    yield glib
    glib.mublis_b200_set_form(b"s", b"plain")


def _edge_gemms(torch):
    """Problems at the edges of the tensor-core grouped path: 1 x 1 x 1,
    k = 0 and alpha = 0 (beta * C only), beta = 0 over a NaN C, rows and
    columns far apart in magnitude (per-row / per-column scaling), ragged
    sizes on both sides of 128 and of the 16 / 32 / 64 column widths, and
    k past one 512-k pack strip."""
    out = []
    for (m, n, k, al, be) in [(1, 1, 1, 1.0, 0.5), (130, 17, 0, 1.0, 0.5), (40, 33, 50, 0.0, 2.0),
                              (129, 65, 300, 1.25, 0.0), (257, 129, 513, 0.75, 0.25),
                              (16, 16, 16, 1.0, 1.0), (8, 200, 31, 1.0, -0.5),
                              (70, 90, 1100, 0.5, 0.5)]:
        a = torch.rand(max(k, 1), m, device="cuda") * 2 - 1
        b = torch.rand(n, max(k, 1), device="cuda") * 2 - 1
        c = torch.rand(n, m, device="cuda") * 2 - 1
        if be == 0.0:
            c.fill_(float("nan"))
        if m == 129:  # op(A) row 3 and op(B) column 5 far from the others
            a[:, 3] *= 2.0 ** 40
            b[5, :] *= 2.0 ** -40
        out.append((GemmProblem(0, 0, m, n, k, al, be, a.data_ptr(), m, b.data_ptr(), max(k, 1),
                                c.data_ptr(), m), (a, b, c)))
    return out


def test_grouped_fp16x3_equals_single_fp16x3_calls(fp16x3):
    """With the FP32 form fp16x3 a group runs on the tensor cores
    (tc_grouped.cu) and gives, problem by problem, the bits of single
    fp16x3 calls (same scaling, split, product order and 256-k windows);
    both stay within 4 k u of plain FP32 calls."""
    torch = pytest.importorskip("torch")
    glib = fp16x3
    probs, keep = make_gemm_set(torch, "s", 96, seed=11, hi=700)
    for pr, k3 in _edge_gemms(torch):
        probs.append(pr)
        keep.append(k3)
    c0 = [c.clone() for _, _, c in keep]
    arr = (GemmProblem * len(probs))(*probs)
    n0 = glib.mublis_b200_launch_count()
    assert glib.mublis_b200_gemm_grouped(b"s", arr, len(probs)) == 0, mb.last_error(glib)
    assert glib.mublis_b200_launch_count() - n0 == 2  # pack + one persistent launch
    grouped = [c.clone() for _, _, c in keep]
    for q, pr in enumerate(probs):
        assert not grouped[q].isnan().any(), (q, pr.m, pr.n, pr.k)
        keep[q][2].copy_(c0[q])
        assert single_call(glib, "s", pr) == 0
        assert torch.equal(grouped[q], keep[q][2]), (q, pr.m, pr.n, pr.k)
    glib.mublis_b200_set_form(b"s", b"plain")
    for q, pr in enumerate(probs):
        keep[q][2].copy_(c0[q])
        assert single_call(glib, "s", pr) == 0
        a, b, _ = keep[q]
        c0n = c0[q].nan_to_num().norm().item() if pr.beta != 0 else 0.0
        den = abs(pr.alpha) * a.norm().item() * b.norm().item() + abs(pr.beta) * c0n
        err = (grouped[q].double() - keep[q][2].double()).norm().item() / max(den, 1e-300)
        assert err <= 4 * max(pr.k, 1) * 2.0 ** -24, (q, pr.m, pr.n, pr.k, err)


def test_grouped_fp16x3_against_oracle(fp16x3):
    torch = pytest.importorskip("torch")
    glib = fp16x3
    m, n, k = 200, 77, 333
    a = orc.fill(k, m, np.float32, 6, 0)   # op(A) = A^T
    b = orc.fill(n, k, np.float32, 6, 1)   # op(B) = B^T
    c0 = orc.fill(m, n, np.float32, 6, 2)
    ta, tb, tc = (torch.from_numpy(x.T.copy()).cuda() for x in (a, b, c0))
    pr = GemmProblem(1, 1, m, n, k, 0.75, 0.25, ta.data_ptr(), k, tb.data_ptr(), n,
                     tc.data_ptr(), m)
    assert glib.mublis_b200_gemm_grouped(b"s", (GemmProblem * 1)(pr), 1) == 0
    ref = c0.copy(order="F")
    assert orc.restated().oracle_sgemm(1, 1, m, n, k, 0.75, a.ctypes.data, 1, k, b.ctypes.data,
                                       1, n, 0.25, ref.ctypes.data, 1, m) == 0
    got = tc.cpu().numpy().T
    err = np.linalg.norm(got - ref) / (0.75 * np.linalg.norm(a) * np.linalg.norm(b) +
                                       0.25 * np.linalg.norm(c0))
    assert err <= 4 * k * 2.0 ** -24


def test_grouped_fp16x3_plan_replay(fp16x3):
    """A plan in the fp16x3 form captures the two launches; creating it runs
    nothing (C unchanged) and its replay equals a direct grouped call."""
    torch = pytest.importorskip("torch")
    glib = fp16x3
    probs, keep = make_gemm_set(torch, "s", 64, seed=13)
    c0 = [c.clone() for _, _, c in keep]
    arr = (GemmProblem * len(probs))(*probs)
    plan = ctypes.c_void_p()
    assert glib.mublis_b200_plan_gemm_grouped(b"s", arr, len(probs), ctypes.byref(plan)) == 0
    for q in range(len(probs)):
        assert torch.equal(keep[q][2], c0[q])
    assert glib.mublis_b200_plan_run(plan) == 0
    replay = [c.clone() for _, _, c in keep]
    for q in range(len(probs)):
        keep[q][2].copy_(c0[q])
    assert glib.mublis_b200_gemm_grouped(b"s", arr, len(probs)) == 0
    for q in range(len(probs)):
        assert torch.equal(replay[q], keep[q][2])
    assert glib.mublis_b200_plan_destroy(plan) == 0
