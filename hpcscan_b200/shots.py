"""Shot-parallel runs over several GPUs: one process per GPU (torch.distributed), each with its
share of a survey's shots in one `Batch` on its own GPU.

Shots are independent: a shot's traces and gradient in a batch are bit-identical to those of the
same shot alone (the batch only shares launches), so a survey split over ranks gives, shot by
shot, the results of one GPU, and nothing crosses GPUs during the time loop. The survey's
adjoint gradient, the sum over its shots of each shot's gradient on a common grid, ends with one
sum all-reduce (NCCL over NVLink on GPUs; any backend for host tensors).

The reference runs one shot per process (TestCase_Modeling, src/testCase_Modeling.cpp:33-282)
and has no adjoint; this is the multi-GPU form of the batched engine (hpcscan_b200.modeling).
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import torch


def shard_shots(work: Sequence[float], world: int) -> List[List[int]]:
    """Shot indices per rank, balanced by work (e.g. grid points x time steps per shot): the
    longest-processing-time rule, shots taken in decreasing work (ties: lower index first), each
    given to the rank with the least work so far (ties: lower rank); every rank's list in
    increasing shot order. Deterministic, so every rank computes the same partition. Equal
    works give the round robin 0, 1, ..., world - 1, 0, 1, ..."""
    if world < 1:
        raise ValueError(f"world size {world}")
    if any(w < 0 for w in work):
        raise ValueError("negative shot work")
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda i: (-work[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += work[i]
    return [sorted(p) for p in parts]


def my_shots(work: Sequence[float], rank: int, world: int) -> List[int]:
    """This rank's shot indices (shard_shots)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    return shard_shots(work, world)[rank]


def _world(group) -> int:
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return 1
    return dist.get_world_size(group)


def sum_gradients(grads: Sequence[torch.Tensor], group=None,
                  out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """The survey gradient from this rank's per-shot gradients: their FP32 sum in the order
    given (an empty list contributes zeros, for a rank without shots, which then needs `out`
    for the shape), then one sum all-reduce over `group` when a process group with more than one
    rank is initialised. Every rank of the group must call it, in the same order as its other
    collectives."""
    if grads:
        shape = grads[0].shape
        for g in grads[1:]:
            if g.shape != shape:
                raise ValueError("shot gradients on different grids cannot be summed")
        total = grads[0].detach().clone() if out is None else out.copy_(grads[0])
        for g in grads[1:]:
            total.add_(g)
    else:
        if out is None:
            raise ValueError("a rank without shots needs `out` for the gradient's shape")
        total = out.zero_()
    if _world(group) > 1:
        import torch.distributed as dist
        dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
    return total


def survey_gradient(batch, group=None, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """sum_gradients over every shot of a gradient `Batch` (modeling.Batch with gradient=True),
    on the shots' common inner grid (n3, n2, n1); a survey batch (survey=True) already holds
    that sum, which is then all-reduced."""
    if getattr(batch, "survey", False):
        return sum_gradients([batch.survey_gradient_of()], group, out)
    return sum_gradients([batch.gradient_of(i) for i in range(len(batch.states))], group, out)
