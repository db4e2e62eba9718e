"""The batched multi-problem sweep (nw_batch_*) against the one-problem path, on the GPU.

Each problem of a batch (different grid sizes, shot counts and step counts, sorted or not) must get
bitwise the traces and gradient that ``WaveOperatorB200.misfit_gradient`` gives it alone with the
same tuning, checkpoint segment and snapshot kind; the graph-replayed batch must equal the eager
one; and the batch gradient must pass the float64 finite-difference and oracle checks through
those equalities (the one-problem path is checked against the oracle in test_gpu_parity.py).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from nefi_b200 import WaveOperatorB200
from nefi_b200._compat import Domain
from nefi_b200.batched import BatchedFWI, autotune

pytestmark = pytest.mark.gpu

K = 16


def _problem(n, shots, n_t, seed, h=10.0, absorbing="sponge"):
    rng = np.random.default_rng(seed)
    dom = Domain((n, n + 8), ((0.0, n * h), (0.0, (n + 8) * h)))
    src = [[(k + 0.5) * n * h / shots, 1.5 * h] for k in range(shots)]
    rec = [[(i + 0.5) * h, 2.5 * h] for i in range(0, n, 2)]
    op = WaveOperatorB200(dom, src, rec, n_t=n_t, dt_obs=1e-3, f0=12.0, c_max=3200.0, order=4,
                          absorbing=absorbing, absorb_width=8 * h, courant=1.0, grad_mode="checkpoint",
                          checkpoint_every=K)
    x = np.linspace(0, 1, n)[:, None] + np.linspace(0, 1, n + 8)[None, :]
    c = 2000.0 + 600.0 * x / 2 + 80.0 * rng.standard_normal((n, n + 8)) * 0.2
    return op, torch.tensor(np.clip(c, 1500.0, 3100.0))


def _batch(dtype, dev):
    specs = [(40, 2, 61, 0), (64, 3, 95, 1), (33, 1, 40, 2), (56, 5, 95, 3)]  # unsorted step counts
    ops, cs, obs = [], [], []
    for n, shots, n_t, seed in specs:
        op, c = _problem(n, shots, n_t, seed)
        with torch.no_grad():
            d = op({"c": (c * 0.97).to(dtype).to(dev)})
        ops.append(op)
        cs.append(c.to(dtype).to(dev))
        obs.append(d)
    return ops, cs, obs


@pytest.mark.parametrize("snapshot", ["fixed16", "exact"])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_batch_equals_each_problem_alone(dtype, snapshot, cuda_device):
    ops, cs, obs = _batch(dtype, cuda_device)
    tuning = (2, 2, 2, 2, 2, 2)
    bt = BatchedFWI(ops, device=cuda_device, dtype=dtype, segment=K, snapshot=snapshot, tuning=tuning)
    losses, grads = bt.misfit_gradients(cs, obs)
    losses = [float(x) for x in losses]
    grads = [g.clone() for g in grads]
    for i, op in enumerate(ops):
        op.snapshot = snapshot
        op.tuning = tuning
        op._plans.clear()
        loss1, g1 = op.misfit_gradient(cs[i], obs[i])
        assert losses[i] == float(loss1), i
        assert torch.equal(grads[i], g1), i
        assert torch.isfinite(g1).all() and g1.abs().max() > 0


def test_graph_replay_equals_eager_batch(cuda_device):
    ops, cs, obs = _batch(torch.float32, cuda_device)
    bt = BatchedFWI(ops, device=cuda_device, segment=K)
    l0, g0 = bt.misfit_gradients(cs, obs)
    l0 = [float(x) for x in l0]
    g0 = [g.clone() for g in g0]
    bt.capture()
    cs2 = [c * 1.001 for c in cs]  # new inputs through the same graph
    l1, g1 = bt.misfit_gradients(cs2, obs)
    l1 = [float(x) for x in l1]
    g1 = [g.clone() for g in g1]
    bt2 = BatchedFWI(ops, device=cuda_device, segment=K)
    l2, g2 = bt2.misfit_gradients(cs2, obs)
    for i in range(len(ops)):
        assert l1[i] == float(l2[i]) and torch.equal(g1[i], g2[i])
        assert l1[i] != l0[i]
    l3, g3 = bt.misfit_gradients(cs, obs)  # and back: the replay is stateless
    for i in range(len(ops)):
        assert float(l3[i]) == l0[i] and torch.equal(g3[i], g0[i])


def test_autotune_returns_a_valid_tuning(cuda_device):
    ops, cs, obs = _batch(torch.float32, cuda_device)
    tuning, results = autotune(ops, steps=20, device=cuda_device, repeats=1)
    assert len(tuning) == 6 and all(v > 0 for v in tuning)
    assert all(t > 0 for t in results.values())
    bt = BatchedFWI(ops, device=cuda_device, segment=K, tuning=tuning)
    _, g = bt.misfit_gradients(cs, obs)
    assert all(torch.isfinite(x).all() for x in g)


@pytest.mark.parametrize("snapshot", ["fixed16", "exact"])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_pml_problems_in_a_batch_equal_each_problem_alone(dtype, snapshot, cuda_device):
    """PML problems (the reference's default layer) in a batch: the interior box goes through the
    batched launch, the layer through the PML kernel; one interior smaller than a tile (all cells
    through the PML kernel) and a sponge problem share the batch."""
    specs = [(96, 3, 95, 5, "pml"), (40, 2, 61, 6, "pml"), (64, 3, 95, 1, "sponge")]
    ops, cs, obs = [], [], []
    for n, shots, n_t, seed, layer in specs:
        op, c = _problem(n, shots, n_t, seed, absorbing=layer)
        with torch.no_grad():
            obs.append(op({"c": (c * 0.97).to(dtype).to(cuda_device)}))
        ops.append(op)
        cs.append(c.to(dtype).to(cuda_device))
    tuning = (2, 2, 2, 2, 2, 2)
    bt = BatchedFWI(ops, device=cuda_device, dtype=dtype, segment=K, snapshot=snapshot, tuning=tuning)
    losses, grads = bt.misfit_gradients(cs, obs)
    losses = [float(x) for x in losses]
    grads = [g.clone() for g in grads]
    for i, op in enumerate(ops):
        op.snapshot = snapshot
        op.tuning = tuning
        op._plans.clear()
        loss1, g1 = op.misfit_gradient(cs[i], obs[i])
        assert losses[i] == float(loss1), i
        assert torch.equal(grads[i], g1), i
        assert torch.isfinite(g1).all() and g1.abs().max() > 0


def test_pml_batch_graph_replay_equals_eager(cuda_device):
    """The per-problem PML launches are captured with the batched ones: replay equals eager."""
    ops, cs, obs = [], [], []
    for n, shots, n_t, seed, layer in [(96, 2, 61, 7, "pml"), (48, 2, 40, 8, "sponge")]:
        op, c = _problem(n, shots, n_t, seed, absorbing=layer)
        with torch.no_grad():
            obs.append(op({"c": (c * 0.97).float().to(cuda_device)}))
        ops.append(op)
        cs.append(c.float().to(cuda_device))
    bt = BatchedFWI(ops, device=cuda_device, segment=K)
    l0, g0 = bt.misfit_gradients(cs, obs)
    l0 = [float(x) for x in l0]
    g0 = [g.clone() for g in g0]
    bt.capture()
    l1, g1 = bt.misfit_gradients(cs, obs)
    for i in range(len(ops)):
        assert float(l1[i]) == l0[i] and torch.equal(g1[i], g0[i])


def test_fused_misfit_batch_equals_each_problem_alone_and_replays(cuda_device):
    """Band-limited relative misfits (with a trace mute) inside the batch: each problem's loss and
    gradient are bitwise those of misfit_gradient(..., misfit=...) alone, and the captured graph
    replays them, also after the observed data change in place."""
    from nefi_b200.misfit import TraceMisfit

    ops, cs, obs = _batch(torch.float32, cuda_device)
    tuning = (2, 2, 2, 2, 2, 2)
    masks = []
    for d in obs:
        m = torch.ones(d.shape[0], d.shape[1], 1, device=cuda_device)
        m[0, 0] = 0.0
        masks.append(m)
    mfs = [TraceMisfit(1e-3, 40.0, 0.3, True) for _ in ops]
    bt = BatchedFWI(ops, device=cuda_device, segment=K, tuning=tuning, misfits=mfs, masks=masks)
    l0, g0 = bt.misfit_gradients(cs, obs)
    l0 = [float(x) for x in l0]
    g0 = [g.clone() for g in g0]
    for i, op in enumerate(ops):
        op.snapshot = bt.snapshot
        op.tuning = tuning
        op._plans.clear()
        l1, g1 = op.misfit_gradient(cs[i], obs[i], misfit=TraceMisfit(1e-3, 40.0, 0.3, True), mask=masks[i])
        assert l0[i] == float(l1), i
        assert torch.equal(g0[i], g1), i
    bt.capture()
    obs2 = [d * 1.1 for d in obs]  # new observations through the same graph
    l2, g2 = bt.misfit_gradients(cs, obs2)
    l2 = [float(x) for x in l2]
    g2 = [g.clone() for g in g2]
    bt2 = BatchedFWI(ops, device=cuda_device, segment=K, tuning=tuning,
                     misfits=[TraceMisfit(1e-3, 40.0, 0.3, True) for _ in ops], masks=masks)
    l3, g3 = bt2.misfit_gradients(cs, obs2)
    for i in range(len(ops)):
        assert l2[i] == float(l3[i]) and torch.equal(g2[i], g3[i]), i
        assert l2[i] != l0[i]
