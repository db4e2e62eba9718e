"""Shot-parallel FWI gradients over several GPUs (one process per GPU, ``torch.distributed``).

Shots are independent until the gradient: each rank runs the forward and adjoint sweeps of its
contiguous share of the sources, and the only exchange is one all-reduce (sum) of the float64
gradient and of the loss per FWI iteration, over NCCL on NVLink/NVSwitch (gloo on CPU for tests).
There is no data-path collective and no domain decomposition: the largest configuration fits one
GPU. This replaces nothing in the reference, whose operators run every shot in one process
(nefi/physics/wave.py:742-750); the sum it returns is the same gradient.
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def shard_slice(n_items: int, rank: int, world: int) -> slice:
    """Contiguous balanced share of ``n_items`` for ``rank`` of ``world``: the first
    ``n_items % world`` ranks take one extra item, so shares differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"invalid rank {rank} of world {world}")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return slice(lo, lo + base + (1 if rank < extra else 0))


def shot_subset(op, sl: slice):
    """A copy of the FWI operator ``op`` restricted to the sources ``op.sources[sl]`` (same grid,
    receivers, time axis, absorbing layer and gradient settings)."""
    from .operators import WaveOperatorB200

    sub = WaveOperatorB200(op.domain, op.sources[sl], op.receivers, f0=op.f0, t0=op.t0,
                           amplitude=op.amplitude, field=op.primary, source_batch=op.source_batch,
                           **op._kwargs())
    if getattr(op, "tuning", None) is not None:
        sub.tuning = op.tuning
    return sub


def misfit_gradient_sharded(op, c: torch.Tensor, observed: torch.Tensor, group=None):
    """``(J, dJ/dc)`` of ``J = 1/2 ||F(c) - observed||^2`` over all of ``op``'s shots, each rank
    computing its share (``shard_slice``) and the float64 sums all-reduced over ``group``.
    Every rank must call it with the same ``c`` and ``observed``; every rank returns the total."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    sl = shard_slice(op.n_sources, rank, world)
    if sl.stop > sl.start:
        loss, grad = shot_subset(op, sl).misfit_gradient(c, observed[sl])
    else:  # more ranks than shots: contribute zeros to the same collectives
        loss = torch.zeros((), dtype=torch.float64, device=c.device)
        grad = torch.zeros(c.shape, dtype=torch.float64, device=c.device)
    if world > 1:
        dist.all_reduce(grad, group=group)
        dist.all_reduce(loss, group=group)
    return loss, grad


def problem_shards(costs, world: int) -> list[list[int]]:
    """Whole problems of a batch over ``world`` ranks, balanced by cost (for FWI: shots x padded cells
    x steps): largest first, each to the rank with the least cost so far (ties to the lower rank).
    Deterministic, so every rank computes the same assignment; returns each rank's problem indices
    in ascending order."""
    if world < 1:
        raise ValueError(f"invalid world size {world}")
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(x) for x in out]


def fwi_cost(op) -> float:
    """Work of one FWI gradient of ``op``: shots x padded cells x steps (forward + adjoint alike)."""
    cells = 1
    for p in op.grid.padded_shape:
        cells *= int(p)
    return float(op.n_sources) * cells * int(op.n_steps)
