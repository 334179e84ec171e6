"""Shot-parallel plumbing on CPU (hpcscan_b200.shots): the deterministic work-balanced partition
of a survey over ranks, and the survey gradient's sum all-reduce with gloo ranks started as
torchrun would start them (world sizes 2 and 3, one rank without shots)."""
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

from hpcscan_b200.shots import my_shots, shard_shots, sum_gradients  # noqa: E402


def test_partition_covers_every_shot_once():
    work = [float(n ** 3) for n in (128, 320, 200, 200, 150, 290, 131)]
    for world in (1, 2, 3, 4, 8, 10):
        parts = shard_shots(work, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(work)))
        assert all(p == sorted(p) for p in parts)
        assert [my_shots(work, r, world) for r in range(world)] == parts


def test_equal_work_is_round_robin():
    assert shard_shots([1.0] * 7, 3) == [[0, 3, 6], [1, 4], [2, 5]]
    assert shard_shots([1.0] * 16, 8) == [[r, r + 8] for r in range(8)]


def test_uneven_survey_is_balanced():
    # the batched-modelling survey: 64 cubes 128^3 .. 320^3
    sizes = [128 + round(192 * s / 63) for s in range(64)]
    work = [float(n ** 3) for n in sizes]
    for world in (2, 4, 8):
        loads = [sum(work[i] for i in p) for p in shard_shots(work, world)]
        assert max(loads) / (sum(work) / world) < 1.03, (world, loads)


def test_bad_arguments():
    with pytest.raises(ValueError):
        shard_shots([1.0], 0)
    with pytest.raises(ValueError):
        shard_shots([-1.0], 2)
    with pytest.raises(ValueError):
        my_shots([1.0], 2, 2)


def test_single_process_sum_is_ordered_fp32():
    import torch
    g = [torch.full((3, 4), 0.1, dtype=torch.float32), torch.full((3, 4), 0.2, dtype=torch.float32),
         torch.full((3, 4), 0.3, dtype=torch.float32)]
    want = (g[0] + g[1]) + g[2]
    assert torch.equal(sum_gradients(g), want)
    with pytest.raises(ValueError):
        sum_gradients([torch.zeros(2), torch.zeros(3)])
    with pytest.raises(ValueError):
        sum_gradients([])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shot_grad(s):
    import torch
    # exactly representable values, so the sum does not depend on the reduction order
    return torch.arange(24, dtype=torch.float32).reshape(2, 3, 4) * float(s + 1)


def _rank_main(rank, world, port, nshot, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = my_shots([1.0] * nshot, rank, world)
        total = sum_gradients([_shot_grad(s) for s in mine], out=torch.empty(2, 3, 4))
        out.put((rank, mine, total.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nshot", [(2, 5), (3, 2)])
def test_survey_gradient_all_reduce_over_gloo_ranks(world, nshot):
    import torch
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nshot, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    want = sum(_shot_grad(s) for s in range(nshot))
    assert sorted(s for _, mine, _ in got for s in mine) == list(range(nshot))
    for rank, mine, total in got:
        assert torch.equal(torch.tensor(total), want), rank
    if world > nshot:
        assert any(not mine for _, mine, _ in got)          # a rank without shots took part
