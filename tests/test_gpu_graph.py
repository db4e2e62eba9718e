"""The whole FWI gradient recorded as one CUDA graph (``WaveOperatorB200.gradient_graph``): every
replay gives bitwise ``misfit_gradient``'s loss and gradient, for each storage mode (full history,
uniform checkpoints with exact and 16-bit snapshots, binomial checkpointing, the PML with its
second stream), for new inputs written in with ``run``, and a corrupted snapshot pool still raises,
after the replay instead of during the capture."""

from __future__ import annotations

import pytest
import torch

from conftest import load_golden
from nefi_b200._compat import SolverError
from test_gpu_parity import make_op

pytestmark = pytest.mark.gpu

MODES = [
    ("fwi_o4_sponge", dict(grad_mode="autograd")),
    ("fwi_o4_sponge", dict(grad_mode="checkpoint", checkpoint_every=10)),
    ("fwi_o4_sponge", dict(grad_mode="checkpoint", checkpoint_every=10, snapshot="delta16")),
    ("fwi_o4_sponge", dict(grad_mode="checkpoint", checkpoint_every=8, checkpoint_slots=2, snapshot="delta16")),
    ("fwi_o4_pml", dict(grad_mode="autograd")),
    ("fwi_o4_pml", dict(grad_mode="checkpoint", checkpoint_every=10, snapshot="fixed16")),
]


def _inputs(case, dev, op, scale=1.0):
    c = torch.tensor(case["c"], dtype=torch.float32, device=dev) * scale
    with torch.no_grad():
        obs = op({"c": c * 1.03})  # data of a slightly faster model
    return c, obs


@pytest.mark.parametrize("name,kw", MODES)
def test_graph_replay_is_bitwise_misfit_gradient(name, kw, cuda_device):
    case = load_golden(name)
    op = make_op(case, **kw)
    c, obs = _inputs(case, cuda_device, op)
    loss0, g0 = op.misfit_gradient(c, obs)
    graph = op.gradient_graph(c, obs, events=True)
    assert graph.launches > 0
    assert graph.checks_status == (kw.get("snapshot", "exact") != "exact")
    for _ in range(2):
        graph.replay()
        graph.check()
        assert torch.equal(graph.loss, loss0) and torch.equal(graph.grad, g0)
    assert graph.events["fwd0"].elapsed_time(graph.events["fwd1"]) > 0
    # new inputs through run(): the same as a fresh misfit_gradient of them
    c2 = c * 0.99
    loss1, g1 = op.misfit_gradient(c2, obs)
    loss2, g2 = graph.run(c2, obs)
    assert torch.equal(loss2, loss1) and torch.equal(g2, g1)
    graph.release()


def test_graph_replay_reports_a_corrupted_snapshot(cuda_device):
    """Host-side fault injection: NaN written into the graph's snapshot pool between replays must
    surface as SolverError from check() (or run()), and the graph must work again afterwards."""
    case = load_golden("fwi_o4_sponge")
    op = make_op(case, grad_mode="checkpoint", checkpoint_every=10, snapshot="delta16")
    c, obs = _inputs(case, cuda_device, op)
    loss0, g0 = op.misfit_gradient(c, obs)
    graph = op.gradient_graph(c, obs)
    graph.replay()
    graph.check()
    # poison the graph's snapshot pool: the forward re-encodes it on each replay, so corrupt the
    # inputs instead, which makes the forward diverge into non-finite snapshots
    bad = c.clone()
    bad[5, 5] = float("inf")
    graph.c.copy_(bad)
    graph.replay()
    with pytest.raises(SolverError, match="non-finite"):
        graph.check()
    loss1, g1 = graph.run(c, obs)
    assert torch.equal(loss1, loss0) and torch.equal(g1, g0)
    graph.release()
