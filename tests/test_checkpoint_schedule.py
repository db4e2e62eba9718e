"""Binomial checkpointing over segments (nefi_b200/plan.py): the schedule the adjoint executes,
simulated on the host. Every segment is reversed exactly once, last to first, from its own start
state; no more slots are used than given; the forward steps it costs are the binomial minimum of
Griewank and Walther's revolve, checked against an exhaustive search on small cases."""

from __future__ import annotations

import math
from functools import lru_cache

import pytest

from nefi_b200.plan import (ADVANCE, RESTORE, TAKE, YOUTURN, binomial_advances, binomial_schedule,
                            binomial_steps, schedule_advances, sweep_readvance)


@lru_cache(None)
def _exhaustive(l: int, s: int) -> int:
    """Fewest advances that reverse l segments from a stored start with s free slots, by exhaustive
    search over the position of the next snapshot (the model revolve's formula solves)."""
    if l <= 1:
        return 0
    if s == 0:
        return l * (l - 1) // 2
    return min(j + _exhaustive(l - j, s - 1) + _exhaustive(j, s) for j in range(1, l))


@pytest.mark.parametrize("c", range(1, 7))
def test_binomial_formula_is_the_exhaustive_minimum(c):
    for l in range(1, 60):
        assert binomial_advances(l, c) == _exhaustive(l, c - 1), (l, c)


def simulate(n_seg: int, n_slots: int):
    """Run the schedule on a model of the ring and the slots; returns the segments in the order they
    were reversed and the number of segments advanced by the adjoint."""
    sweep_slot, actions = binomial_schedule(n_seg, n_slots)
    slots = {}
    for j, k in enumerate(sweep_slot):  # the forward sweep: every segment start passes by once
        if k >= 0:
            assert 0 <= k < n_slots
            slots[k] = j
    assert sweep_slot[0] >= 0  # segment 0's start is always kept
    cur, reversed_, advanced = None, [], 0
    for op, x, y in actions:
        if op == RESTORE:
            assert slots.get(x) == y, "a slot decodes the state it holds"
            cur = y
        elif op == ADVANCE:
            assert cur == x and y > x
            advanced += y - x
            cur = y
        elif op == TAKE:
            assert 0 <= x < n_slots and cur == y
            slots[x] = y
        elif op == YOUTURN:
            assert cur == x, "a segment is recomputed from its own start"
            reversed_.append(x)
            cur = None
        else:
            raise AssertionError(op)
    return reversed_, advanced


@pytest.mark.parametrize("n_seg,n_slots", [(1, 1), (2, 1), (7, 7), (10, 3), (20, 1), (40, 5), (89, 20),
                                           (200, 12), (63, 63), (64, 2), (150, 40)])
def test_schedule_reverses_every_segment_once_at_the_binomial_cost(n_seg, n_slots):
    reversed_, advanced = simulate(n_seg, n_slots)
    assert reversed_ == list(range(n_seg - 1, -1, -1))
    sweep_slot, actions = binomial_schedule(n_seg, n_slots)
    # the adjoint advances: revolve's minimum less the sweep's n_seg - 1, plus the segments the first
    # reversal re-advances because the sweep ran on to the last step for the traces
    assert advanced == binomial_advances(n_seg, n_slots) - (n_seg - 1) + sweep_readvance(n_seg, n_slots)
    assert schedule_advances(n_seg, sweep_slot, actions) == binomial_advances(n_seg, n_slots) + \
        sweep_readvance(n_seg, n_slots)
    if n_slots >= n_seg:
        assert advanced == 0  # a snapshot per segment: no advance at all, the uniform scheme


def test_fewer_slots_cost_more_steps_and_enough_slots_cost_two_sweeps():
    n = 8000
    costs = [binomial_steps(n, 90, s) for s in (89, 60, 30, 15, 8, 4)]
    assert costs[0] == 2 * n
    assert all(a <= b for a, b in zip(costs, costs[1:]))
    # the repetition number grows slowly: 30 slots for 89 segments costs under one extra sweep
    assert costs[2] < 3 * n


def test_storage_plan_switches_to_binomial_checkpointing_under_a_small_budget():
    """With a budget below a snapshot per segment at any segment length, the plan keeps fewer slots
    and the schedule's extra forward steps; with enough memory it keeps the uniform scheme."""
    import torch

    from nefi_b200 import WaveOperatorB200
    from nefi_b200._compat import Domain
    from nefi_b200.plan import plan_storage

    n, h = 64, 10.0
    op = WaveOperatorB200(Domain((n, n), ((0.0, n * h), (0.0, n * h))), [[320.0, 15.0]], [[320.0, 25.0]],
                          n_t=901, dt_obs=1e-3, f0=10.0, c_max=2500.0, absorbing="sponge", absorb_width=100.0,
                          courant=1.0)
    plan = op._plan(torch.device("cpu"), torch.float32)
    lvl = plan.level_bytes(1)
    big = plan_storage(plan, 1, op.n_steps, "checkpoint", None, "delta16", None)
    assert big == ("checkpoint", math.ceil(math.sqrt(op.n_steps)))
    snap1 = plan.snapshot_bytes(1, 1, 4)
    budget = 12 * lvl + 6 * snap1  # far below a snapshot per segment at any segment length
    mode = plan_storage(plan, 1, op.n_steps, "checkpoint", None, "delta16", budget)
    assert len(mode) == 3 and mode[2] < -(-op.n_steps // mode[1])
    k, slots = mode[1], mode[2]
    assert slots * snap1 + (k + 3) * lvl <= budget
    fixed = plan_storage(plan, 1, op.n_steps, "checkpoint", 10, "exact", None, checkpoint_slots=4)
    assert fixed == ("checkpoint", 10, 4)
