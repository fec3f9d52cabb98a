"""The request server (continuous batching across host threads).

Each request's result must be the same alone and in the mix: every call of a
mixed set (small and large SGEMM, DGEMM, SSYRK, DTRSM) is first run alone on
the direct path, then the same calls are issued concurrently from 16 host
threads through the attached server, and each output is compared with its
alone result (normwise relative error <= 4 * k * u; the server's coalesced
launches may sum in another order).  The server statistics must show that
small requests were coalesced.
"""
import ctypes
import threading

import numpy as np
import pytest

import mublis_b200 as mb

pytestmark = pytest.mark.gpu


ServerConfig, ServerStats = mb.ServerConfig, mb.ServerStats


def declare_server(lib):
    """The package declares the server entry points; kept for callers."""
    return lib


def make_calls(torch, count, seed, large=(768, 1024)):
    rng = np.random.default_rng(seed)
    calls = []
    for q in range(count):
        kind = rng.choice(["sgemm", "dgemm", "ssyrk", "dtrsm"], p=[0.6, 0.2, 0.1, 0.1])
        if rng.random() < 0.85:
            n1, n2, n3 = (int(x) for x in np.floor(np.exp(rng.uniform(np.log(32), np.log(257), 3))))
        else:
            n1 = n2 = n3 = int(rng.choice(list(large)))
        dt = torch.float32 if kind[0] == "s" else torch.float64
        if kind.endswith("gemm"):
            m, n, k = n1, n2, n3
            ops = [torch.rand(k, m, dtype=dt, device="cuda") - 0.5,
                   torch.rand(n, k, dtype=dt, device="cuda") - 0.5,
                   torch.rand(n, m, dtype=dt, device="cuda") - 0.5]
            calls.append(dict(kind=kind, m=m, n=n, k=k, ops=ops))
        elif kind == "ssyrk":
            n, k = n1, n3
            ops = [torch.rand(k, n, dtype=dt, device="cuda") - 0.5,
                   torch.rand(n, n, dtype=dt, device="cuda") - 0.5]
            calls.append(dict(kind=kind, m=n, n=n, k=k, ops=ops))
        else:
            m, n = n1, n2
            a = (torch.rand(m, m, dtype=dt, device="cuda") - 0.5) / m
            a.diagonal().copy_(torch.rand(m, dtype=dt, device="cuda") + 1)
            calls.append(dict(kind=kind, m=m, n=n, k=m,
                              ops=[a, torch.rand(n, m, dtype=dt, device="cuda") - 0.5]))
    return calls


def issue(lib, c):
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    o = c["ops"]
    if c["kind"] == "sgemm":
        lib.cblas_sgemm(mb.COL, mb.NO_TRANS, mb.NO_TRANS, c["m"], c["n"], c["k"], 0.75, p(o[0]),
                        c["m"], p(o[1]), c["k"], 0.25, p(o[2]), c["m"])
    elif c["kind"] == "dgemm":
        lib.cblas_dgemm(mb.COL, mb.NO_TRANS, mb.NO_TRANS, c["m"], c["n"], c["k"], 0.75, p(o[0]),
                        c["m"], p(o[1]), c["k"], 0.25, p(o[2]), c["m"])
    elif c["kind"] == "ssyrk":
        lib.cblas_ssyrk(mb.COL, mb.LOWER, mb.NO_TRANS, c["n"], c["k"], 0.75, p(o[0]), c["n"],
                        0.25, p(o[1]), c["n"])
    else:
        lib.cblas_dtrsm(mb.COL, mb.LEFT, mb.LOWER, mb.NO_TRANS, mb.NON_UNIT, c["m"], c["n"], 0.75,
                        p(o[0]), c["m"], p(o[1]), c["m"])


@pytest.mark.parametrize("forms", ["plain", "auto"])
def test_results_are_the_same_alone_and_in_the_mix(forms):
    """forms "auto": the large requests run the tensor-core forms the policy
    picks (bf16x6 for FP32 from 512, the modular Ozaki form for FP64 from
    2048^2), alone and in the mix."""
    torch = pytest.importorskip("torch")
    lib = declare_server(mb.load())
    assert lib.mublis_b200_init() == 0
    for p in (b"s", b"d"):
        lib.mublis_b200_set_form(p, forms.encode())
    calls = make_calls(torch, 96, seed=2,
                       large=(768, 1024) if forms == "plain" else (768, 1024, 2048))
    out_idx = lambda c: 1 if c["kind"] in ("ssyrk", "dtrsm") else 2  # noqa: E731
    initial = [c["ops"][out_idx(c)].clone() for c in calls]

    # alone: direct path, one call at a time
    alone = []
    for c, init in zip(calls, initial):
        c["ops"][out_idx(c)].copy_(init)
        torch.cuda.synchronize()
        issue(lib, c)
        alone.append(c["ops"][out_idx(c)].clone())
        c["ops"][out_idx(c)].copy_(init)
    torch.cuda.synchronize()

    # in the mix: 16 host threads through the attached server
    # Forms left to the library default set above (NULL in the config).
    cfg = ServerConfig(hbm_budget_bytes=8 << 30, streams=4, batch_window_us=200,
                       small_max_dim=512, max_batch=4096, sform=None, dform=None)
    srv = ctypes.c_void_p()
    assert lib.mublis_b200_server_create(ctypes.byref(cfg), ctypes.byref(srv)) == 0
    assert lib.mublis_b200_server_attach(srv) == 0
    try:
        chunks = [calls[t::16] for t in range(16)]
        errors = []

        def worker(chunk):
            try:
                for c in chunk:
                    issue(lib, c)
            except Exception as e:  # noqa: BLE001
                errors.append(e)

        threads = [threading.Thread(target=worker, args=(ch,)) for ch in chunks]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors
        st = ServerStats()
        assert lib.mublis_b200_server_stats(srv, ctypes.byref(st)) == 0
    finally:
        lib.mublis_b200_server_attach(None)
        lib.mublis_b200_server_destroy(srv)
        for p in (b"s", b"d"):
            lib.mublis_b200_set_form(p, b"plain")
    torch.cuda.synchronize()

    assert st.completed == len(calls)
    assert st.batches >= 1 and st.batched_requests >= 2  # small requests were coalesced
    assert st.p99_latency_s >= st.p50_latency_s > 0
    for c, ref, init in zip(calls, alone, initial):
        got = c["ops"][out_idx(c)].double()
        u = 2.0 ** -24 if c["kind"][0] == "s" else 2.0 ** -53
        if c["kind"] == "dtrsm":
            err = (got - ref.double()).norm().item() / ref.double().norm().item()
        else:
            o = c["ops"]
            den = 0.75 * o[0].double().norm().item() * (o[0] if c["kind"] == "ssyrk" else o[1]).double().norm().item() \
                + 0.25 * init.double().norm().item()
            err = (got - ref.double()).norm().item() / den
        assert err <= 4 * max(c["k"], 1) * u, (c["kind"], c["m"], c["n"], c["k"], err)


def test_server_alloc_respects_the_hbm_budget():
    lib = declare_server(mb.load())
    assert lib.mublis_b200_init() == 0
    cfg = ServerConfig(hbm_budget_bytes=64 << 20, streams=2)
    srv = ctypes.c_void_p()
    assert lib.mublis_b200_server_create(ctypes.byref(cfg), ctypes.byref(srv)) == 0
    try:
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        assert lib.mublis_b200_server_alloc(srv, 48 << 20, ctypes.byref(a)) == 0
        assert lib.mublis_b200_server_alloc(srv, 32 << 20, ctypes.byref(b)) == 3  # over budget
        assert lib.mublis_b200_server_free(srv, a) == 0
        assert lib.mublis_b200_server_alloc(srv, 32 << 20, ctypes.byref(b)) == 0
        assert lib.mublis_b200_server_free(srv, b) == 0
    finally:
        lib.mublis_b200_server_destroy(srv)
