"""Shot-parallel FWI gradient on gloo ranks (CPU).

``misfit_gradient_sharded`` splits the shots over the ranks and all-reduces the float64 loss and
gradient. Here each rank's share runs through the CPU oracle (a test double standing in for the
device sweep, which needs a GPU); the all-reduced result must equal the one-process gradient over
all shots, for an even and an uneven split and for more ranks than shots."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_golden, rel_l2
from nefi_b200 import WaveOperatorB200, distributed
from nefi_b200._compat import Domain

CASE = "fwi_o4_sponge"


@pytest.mark.parametrize("n,world", [(16, 2), (5, 2), (3, 4), (1, 2), (0, 3)])
def test_shard_slices_partition_the_shots(n, world):
    parts = [distributed.shard_slice(n, r, world) for r in range(world)]
    assert parts[0].start == 0 and parts[-1].stop == n
    assert all(parts[r].stop == parts[r + 1].start for r in range(world - 1))
    sizes = [p.stop - p.start for p in parts]
    assert max(sizes) - min(sizes) <= 1


def _case_op(case, sources=None):
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    src = case["sources"] if sources is None else sources
    return WaveOperatorB200(dom, src, case["receivers"], grad_mode="autograd", **case["kw"])


def _oracle_misfit(case, sources, c, observed):
    """(J, dJ/dc) over ``sources`` through the float64 oracle."""
    import oracle

    orc = oracle.OracleWave(case["shape"], case["extent"], case["receivers"], sources=sources, **case["kw"])
    tr, _ = orc.fwi(c, None, dtype=np.float64)
    r = tr - observed
    _, g = orc.fwi(c, r, dtype=np.float64)
    return 0.5 * float((r * r).sum()), g


def _observed(case):
    """Synthetic observed data: traces of a 2 % slower model, so the residual is not zero."""
    import oracle

    orc = oracle.OracleWave(case["shape"], case["extent"], case["receivers"], sources=case["sources"], **case["kw"])
    tr, _ = orc.fwi(np.asarray(case["c"]) * 0.98, None, dtype=np.float64)
    return tr


def _worker(rank, world, port, sources, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = load_golden(CASE)
        op = _case_op(case, sources)
        c = torch.tensor(case["c"], dtype=torch.float64)
        all_obs = _observed({**case, "sources": sources})
        obs = torch.tensor(all_obs)

        def misfit_gradient(self, cc, observed):  # the device sweep's CPU stand-in
            loss, g = _oracle_misfit(case, self.sources.numpy(), cc.numpy(), observed.numpy())
            return torch.tensor(loss, dtype=torch.float64), torch.tensor(g, dtype=torch.float64)

        WaveOperatorB200.misfit_gradient = misfit_gradient
        loss, grad = distributed.misfit_gradient_sharded(op, c, obs)
        queue.put((rank, float(loss), grad.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n_src,world", [(4, 2), (3, 2), (2, 3)])
def test_sharded_gradient_equals_one_process_gradient(n_src, world):
    case = load_golden(CASE)
    L = case["extent"][0][1] - case["extent"][0][0]
    z = float(case["sources"][0][1])
    sources = np.stack([(np.arange(n_src) + 0.5) * L / n_src, np.full(n_src, z)], 1)
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sources, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref_loss, ref_grad = _oracle_misfit(case, sources, np.asarray(case["c"]), _observed({**case, "sources": sources}))
    for _, loss, grad in results:  # every rank holds the total
        assert abs(loss - ref_loss) <= 1e-12 * abs(ref_loss)
        assert rel_l2(grad, ref_grad) < 1e-12


def test_problem_shards_cover_every_problem_once_and_balance():
    from nefi_b200.distributed import problem_shards

    rng = np.random.default_rng(3)
    costs = rng.integers(1, 100, size=37).astype(float)
    for world in (1, 2, 3, 8, 40):
        shards = problem_shards(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        # largest-first greedy: the spread never exceeds the largest single cost
        assert max(loads) - min(loads) <= costs.max() + 1e-9
        assert shards == problem_shards(list(costs), world)  # deterministic


def _shard_worker(rank, world, port, q):
    import torch.distributed as dist

    from nefi_b200.distributed import problem_shards

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        costs = [5.0, 1.0, 7.0, 3.0, 3.0, 2.0]
        mine = problem_shards(costs, world)[rank]
        t = torch.tensor([float(len(mine)), sum(costs[i] for i in mine)], dtype=torch.float64)
        dist.all_reduce(t)
        q.put((rank, mine, t.tolist()))
    finally:
        dist.destroy_process_group()


def test_problem_shards_agree_across_gloo_ranks():
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = dict((r, (m, t)) for r, m, t in res)
    assert sorted(got[0][0] + got[1][0]) == list(range(6))
    assert got[0][1] == [6.0, 21.0] and got[1][1] == [6.0, 21.0]
