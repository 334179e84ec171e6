"""The multi-rank plumbing of bench.py on CPU: two gloo ranks, as torchrun would start them.

bench.py runs one replica of the propagator per GPU ("replicas only": one grid does not
shard); the only cross-rank steps are the barrier and the max over ranks of the timings, and
value = all ranks' points / that maximum. The reference arm prints from rank 0 only.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r timed (r + 1) ms for the whole run and (10 - r) ms for the kernel
        ms, kern = bench.max_over_ranks(dist, [rank + 1.0, 10.0 - rank], "cpu")
        value = bench.job_gpoints(world, 1_000_000, 100, ms * 1e-3)
        out.put((rank, ms, kern, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_value_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, kern, value in got:
        assert (ms, kern) == (2.0, 10.0)                 # the max over both ranks, on every rank
        assert value == pytest.approx(2 * 1_000_000 * 100 / 2e-3 / 1e9)   # 100 GPoint/s


def test_single_process_keeps_its_own_timings():
    import bench
    assert bench.max_over_ranks(None, [3.0, 4.0], "cpu") == [3.0, 4.0]


def test_reference_arm_prints_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "run_reference_cpu", lambda *a: called.append(a))
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.reference_arm(_args())
    assert buf.getvalue() == "" and not called


def _args():
    import argparse
    return argparse.Namespace(gpus=2, steps=3, warmup=3, impl="reference", size=64, order=8,
                              e2e_steps=0, cpu_steps=3, no_cpu=True)
