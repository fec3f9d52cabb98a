"""bench.py's multi-replica arithmetic on world-size-2 gloo ranks (CPU).

`bench.py --gpus N` runs one replica per GPU under torchrun: every rank
times its own replica, the job's time is the slowest rank's (all-reduce
MAX), the whole-job value is N x the per-rank flops over that time, and only
rank 0 prints.  Here two CPU processes with the gloo backend stand in for
the ranks (no GPU involved), each reporting a different time.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        own_ms = 10.0 * (rank + 1)
        ms = bench.max_over_ranks(dist, torch, own_ms, world, device="cpu")
        value = bench.whole_job_tflops(1e12, world, ms)
        args = type("A", (), {"steps": 1, "warmup": 3, "n": 1024})()
        buf = io.StringIO()
        if rank != 0:  # the reference arm: ranks other than 0 do nothing and print nothing
            with redirect_stdout(buf):
                bench.run_reference_arm(args, rank, world)
        out.put((rank, ms, value, buf.getvalue()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]  # both ranks see the max
    for _, _, value, printed in res:
        assert value == pytest.approx(2 * 1e12 / 20e-3 / 1e12)  # 100 TF/s whole job
        assert printed == ""


def test_single_rank_is_unchanged():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(None, None, 12.5, 1) == 12.5
    assert bench.whole_job_tflops(2e12, 1, 10.0) == pytest.approx(200.0)
