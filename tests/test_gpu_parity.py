"""GPU parity of the CUDA propagator (through the C ABI) against the reference's golden vectors
and the CPU oracle.

Tolerances (relative L2):
  float64 device run vs reference float64: traces 1e-11, gradients 1e-10 (rounding only);
  float32 device run vs reference float32: traces 1e-5, gradients 1e-4 (the stated FP32 bar);
  float32 device run vs the float64 oracle: traces 1e-5, gradients 1e-4.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import cotangent, full_trace_shape, golden_names, load_golden, oracle_for, rel_l2
from nefi_b200 import WaveInitialConditionOperatorB200, WaveOperatorB200
from nefi_b200._compat import Domain, OperatorError, SolverError

pytestmark = pytest.mark.gpu

FWI = golden_names("fwi")
PAT = golden_names("pat")


def make_op(case, tuning=None, **over):
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    kw = {**case["kw"], "grad_mode": "autograd", **over}
    if case["kind"] == "fwi":
        op = WaveOperatorB200(dom, case["sources"], case["receivers"], **kw)
    else:
        op = WaveInitialConditionOperatorB200(dom, case["receivers"], c=torch.tensor(case["c"]), **kw)
    if tuning is not None:
        op.tuning = tuning
    return op


def run_fwi(case, dtype, dev, **over):
    op = make_op(case, **over)
    c = torch.tensor(case["c"], dtype=dtype, device=dev, requires_grad=True)
    tr = op({"c": c})
    g = torch.tensor(cotangent(tr.shape, case["seed"]), dtype=dtype, device=dev)
    (gc,) = torch.autograd.grad((tr * g).sum(), c)
    return tr.detach()[:, :: case["rec_stride"]].cpu().numpy(), gc.cpu().numpy()


def run_pat(case, dtype, dev, with_c=False, **over):
    op = make_op(case, **over)
    p0 = torch.tensor(case["p0"], dtype=dtype, device=dev, requires_grad=True)
    if with_c:
        c = torch.tensor(case["c"], dtype=dtype, device=dev, requires_grad=True)
        tr = op.with_speed(p0, c)
    else:
        tr = op({"p0": p0})
    g = torch.tensor(cotangent(tr.shape, case["seed"]), dtype=dtype, device=dev)
    if with_c:
        gp, gc = torch.autograd.grad((tr * g).sum(), (p0, c))
        return tr.detach().cpu().numpy(), gp.cpu().numpy(), gc.cpu().numpy()
    (gp,) = torch.autograd.grad((tr * g).sum(), p0)
    return tr.detach().cpu().numpy(), gp.cpu().numpy(), None


@pytest.mark.parametrize("name", FWI)
def test_fwi_float64_matches_reference(name, cuda_device):
    case = load_golden(name)
    tr, gc = run_fwi(case, torch.float64, cuda_device)
    assert rel_l2(tr, case["traces_f64"]) < 1e-11
    assert rel_l2(gc, case["grad_c_f64"]) < 1e-10


@pytest.mark.parametrize("name", FWI)
def test_fwi_float32_matches_reference_float32(name, cuda_device):
    case = load_golden(name)
    tr, gc = run_fwi(case, torch.float32, cuda_device)
    assert rel_l2(tr, case["traces_f32"]) < 1e-5
    assert rel_l2(gc, case["grad_c_f32"]) < 1e-4
    # and against the float64 oracle
    assert rel_l2(tr, case["traces_f64"]) < 1e-5
    assert rel_l2(gc, case["grad_c_f64"]) < 1e-4


@pytest.mark.parametrize("name", PAT)
def test_pat_float64_matches_reference(name, cuda_device):
    case = load_golden(name)
    tr, gp, _ = run_pat(case, torch.float64, cuda_device)
    assert rel_l2(tr, case["traces_f64"]) < 1e-11
    assert rel_l2(gp, case["grad_p0_f64"]) < 1e-10
    tr2, gp2, gc = run_pat(case, torch.float64, cuda_device, with_c=True)
    assert rel_l2(tr2, case["traces_f64"]) < 1e-11
    assert rel_l2(gp2, case["grad_p0_f64"]) < 1e-10
    assert rel_l2(gc, case["grad_c_f64"]) < 1e-10


@pytest.mark.parametrize("name", PAT)
def test_pat_float32_matches_reference_float32(name, cuda_device):
    case = load_golden(name)
    tr, gp, _ = run_pat(case, torch.float32, cuda_device)
    assert rel_l2(tr, case["traces_f32"]) < 1e-5
    assert rel_l2(gp, case["grad_p0_f32"]) < 1e-4
    _, _, gc = run_pat(case, torch.float32, cuda_device, with_c=True)
    assert rel_l2(gc, case["grad_c_f32"]) < 1e-4


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("name", ["fwi_o4_sponge", "fwi_o4_cerjan", "pat3d_o2_sponge", "fwi_o4_pml",
                                  "fwi_o2_pml_aniso", "pat2d_o4_pml"])
def test_checkpointed_gradient_is_identical_to_full_history(name, dtype, cuda_device):
    case = load_golden(name)
    if case["kind"] == "fwi":
        ref = run_fwi(case, dtype, cuda_device)
        for k in (5, None):
            got = run_fwi(case, dtype, cuda_device, grad_mode="checkpoint", checkpoint_every=k)
            assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    else:
        ref = run_pat(case, dtype, cuda_device)
        got = run_pat(case, dtype, cuda_device, grad_mode="checkpoint", checkpoint_every=7)
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


@pytest.mark.parametrize("slots", [1, 2, 3])
@pytest.mark.parametrize("name", ["fwi_o4_sponge", "fwi_o4_pml", "pat3d_o2_sponge"])
def test_binomial_checkpointing_is_identical_to_full_history(name, slots, cuda_device):
    """Fewer snapshot slots than segments: the adjoint follows the binomial schedule (restores, advances,
    new snapshots) and, with exact snapshots, gives bitwise the full-history traces and gradient."""
    case = load_golden(name)
    if case["kind"] == "fwi":
        ref = run_fwi(case, torch.float32, cuda_device)
        got = run_fwi(case, torch.float32, cuda_device, grad_mode="checkpoint", checkpoint_every=3,
                      checkpoint_slots=slots)
    else:
        ref = run_pat(case, torch.float32, cuda_device)
        got = run_pat(case, torch.float32, cuda_device, grad_mode="checkpoint", checkpoint_every=3,
                      checkpoint_slots=slots)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_binomial_checkpointing_with_16_bit_snapshots(cuda_device):
    case = load_golden("cfg1_128_o4_sponge")
    tr, gc = run_fwi(case, torch.float32, cuda_device, grad_mode="checkpoint", checkpoint_every=40,
                     checkpoint_slots=6, snapshot="delta16")
    assert rel_l2(tr, case["traces_f64"]) < 1e-5
    assert rel_l2(gc, case["grad_c_f64"]) < 1e-4


@pytest.mark.parametrize("snapshot,tol", [("delta16", 1e-4), ("fixed16", 3e-4), ("fp16", 3e-3), ("bf16", 2.5e-2)])
def test_reduced_precision_snapshots_error_is_bounded(snapshot, tol, cuda_device):
    """16-bit snapshots perturb only the recomputed forward field, so the traces stay exact and the
    gradient error is set by the rounding noise of the codec. The seeded white-noise cotangent of
    this fixture excites the grid's shortest wavelengths, where the Laplacian amplifies that noise
    most: delta16 meets the 1e-4 gradient budget (4.4e-5 in a CPU model of the codec), fixed16, fp16
    and bf16 do not (1.8e-4, 2.0e-3, 1.7e-2; 40-step segments, float64 oracle)."""
    case = load_golden("cfg1_128_o4_sponge")
    tr, gc = run_fwi(case, torch.float32, cuda_device, grad_mode="checkpoint", checkpoint_every=40,
                     snapshot=snapshot)
    assert rel_l2(tr, case["traces_f64"]) < 1e-5  # the forward never reads a snapshot
    assert rel_l2(gc, case["grad_c_f64"]) < tol


@pytest.mark.parametrize("absorbing,n", [("sponge", 192), ("pml", 160)])
@pytest.mark.parametrize("snapshot", ["delta16", "fixed16"])
def test_checkpointed_16_bit_gradient_of_a_salt_model_meets_the_budget(absorbing, n, snapshot, cuda_device):
    """The north-star method on the large configuration's model family (layers + a 4500 m/s salt body,
    12 Hz), reduced to a grid a float64 CPU run finishes in seconds: 32 shots, 1000 steps, the default
    ceil(sqrt(N)) = 32-step segments, 16-bit snapshots. The cotangent is the residual of
    1/2 ||d(c0) - d(c_true)||^2 at a smoothed model c0, as an FWI iteration takes it. The float32
    gradient must be within 1e-4 (relative L2) of the float64 oracle's, with the sponge and the PML."""
    import oracle
    from scipy.ndimage import gaussian_filter
    from nefi_b200.workloads import fwi_salt

    w = fwi_salt(n=n, n_shots=32, n_steps=1000)
    kw = {**w.operator_kwargs(), "absorbing": absorbing}
    orc = oracle.OracleWave((n, n), ((0.0, n * w.h), (0.0, n * w.h)), w.receivers, sources=w.sources, **kw)
    oracle.set_threads(max(1, __import__("os").cpu_count() or 1))
    c0 = gaussian_filter(w.c, 6.0)
    obs, _ = orc.fwi(w.c)
    pred, _ = orc.fwi(c0)
    resid = pred - obs
    _, g64 = orc.fwi(c0, resid)
    op = WaveOperatorB200(w.domain, w.sources, w.receivers, grad_mode="checkpoint", snapshot=snapshot, **kw)
    c = torch.tensor(c0, dtype=torch.float32, device=cuda_device, requires_grad=True)
    tr = op({"c": c})
    (gc,) = torch.autograd.grad((tr * torch.tensor(resid, dtype=torch.float32, device=cuda_device)).sum(), c)
    # the forward never reads a snapshot: its traces carry only float32 rounding, which over 1000
    # steps reaches about 1e-5 of the float64 run (1.05e-5 with the PML)
    assert rel_l2(tr.detach().cpu().numpy(), pred) < 3e-5
    err = rel_l2(gc.cpu().numpy(), g64)
    print(f"{absorbing} {snapshot}: float32 checkpointed gradient vs float64 oracle {err:.2e}")
    assert err < 1e-4


@pytest.mark.parametrize("snapshot", ["delta16", "fixed16", "bf16"])
def test_pml_checkpoints_with_16_bit_snapshots(snapshot, cuda_device):
    """The PML's face fields travel through the 16-bit codec with the pressure; the traces stay exact
    and the gradient stays close to the reference's float64 one."""
    case = load_golden("fwi_o4_pml")
    tr, gc = run_fwi(case, torch.float32, cuda_device, grad_mode="checkpoint", checkpoint_every=6,
                     snapshot=snapshot)
    assert rel_l2(tr, case["traces_f64"]) < 1e-5
    assert rel_l2(gc, case["grad_c_f64"]) < {"delta16": 1e-3, "fixed16": 1e-3, "bf16": 3e-2}[snapshot]


def test_runs_are_bitwise_deterministic(cuda_device):
    case = load_golden("fwi_o4_sponge")
    a = run_fwi(case, torch.float32, cuda_device)
    b = run_fwi(case, torch.float32, cuda_device)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_central_finite_differences_float64(cuda_device):
    """The reference's own check (tests/test_physics_wave.py:145-165), on the device."""
    torch.manual_seed(0)
    dom = Domain((16, 16), ((0.0, 1.0), (0.0, 1.0)))
    c = (2.0 + 0.2 * torch.randn(16, 16, dtype=torch.float64)).clamp(1.6, 2.4).to(cuda_device)
    kw = dict(n_t=40, dt_obs=0.01, f0=5.0, c_max=2.5, absorb_width=0.2, absorbing="sponge")
    src, rec = [[0.2, 0.3], [0.2, 0.7]], [[0.8, y] for y in (0.2, 0.4, 0.6, 0.8)]
    w = torch.randn(2, 4, 40, dtype=torch.float64).to(cuda_device)
    grads = []
    for mode, ck in (("autograd", None), ("checkpoint", 5), ("checkpoint", None)):
        op = WaveOperatorB200(dom, src, rec, grad_mode=mode, checkpoint_every=ck, **kw)
        x = c.clone().requires_grad_(True)
        (g,) = torch.autograd.grad((op({"c": x}) * w).sum(), x)
        grads.append(g)
    for g in grads[1:]:
        assert float((g - grads[0]).norm() / grads[0].norm()) < 1e-6
    op = WaveOperatorB200(dom, src, rec, grad_mode="autograd", **kw)
    for seed in range(4):
        e = torch.randn(16, 16, dtype=torch.float64, generator=torch.Generator().manual_seed(seed)).to(cuda_device)
        eps = 1e-6
        fd = float((op({"c": c + eps * e}) * w).sum()) - float((op({"c": c - eps * e}) * w).sum())
        fd /= 2 * eps
        assert abs(fd - float((grads[0] * e).sum())) < 1e-6 * max(1.0, abs(fd))


def test_pat_adjoint_identity_and_linearity_float64(cuda_device):
    """<A a, y> = <a, A^T y> (tests/test_photoacoustic3d.py:49-59), on the device."""
    case = load_golden("pat3d_o2_sponge")
    op = make_op(case)
    dev, F = cuda_device, torch.float64
    g = torch.Generator().manual_seed(0)
    a = torch.rand(12, 12, 8, dtype=F, generator=g).to(dev)
    b = torch.rand(12, 12, 8, dtype=F, generator=g).to(dev)
    ya, yb = op({"p0": a}), op({"p0": b})
    assert torch.allclose(op({"p0": 2 * a - 0.5 * b}), 2 * ya - 0.5 * yb, atol=1e-10)
    y = torch.randn(ya.shape, dtype=F, generator=g).to(dev)
    x = torch.zeros(12, 12, 8, dtype=F, device=dev, requires_grad=True)
    (adj,) = torch.autograd.grad((op({"p0": x}) * y).sum(), x)
    assert float((ya * y).sum()) == pytest.approx(float((a * adj).sum()), rel=1e-9)


@pytest.mark.parametrize("absorbing", ["pml", "sponge"])
def test_multiresolution_source_batching_and_speed_check(absorbing, cuda_device):
    """tests/test_physics_wave.py:168-189 on the device: a 2x coarser grid gives the same physics
    within 20 %, shot chunks give the same traces, a speed above c_max is refused."""
    dom = Domain((32, 32), ((0.0, 1.0), (0.0, 1.0)))
    src = [[0.1, 0.3], [0.1, 0.5], [0.1, 0.7]]
    rec = [[0.9, y] for y in torch.linspace(0.1, 0.9, 6).tolist()]
    kw = dict(n_t=60, dt_obs=0.016, f0=3.0, c_max=2.5, absorb_width=0.25, absorbing=absorbing)
    op = WaveOperatorB200(dom, src, rec, **kw)
    x = dom.physical_coords(dtype=torch.float64)
    c = (2.0 + 0.2 * torch.exp(-((x - 0.5) ** 2).sum(-1) / 0.02)).to(cuda_device)
    y = op({"c": c})
    assert y.shape == (3, 6, 60) == op.output_shape((32, 32))
    coarse = op.at_resolution((16, 16))
    assert coarse is op.at_resolution((16, 16)) and coarse.grid.shape == (16, 16)
    assert coarse.fidelity_tag == op.fidelity_tag
    xc = dom.at((16, 16)).physical_coords(dtype=torch.float64)
    yc = coarse({"c": (2.0 + 0.2 * torch.exp(-((xc - 0.5) ** 2).sum(-1) / 0.02)).to(cuda_device)})
    assert yc.shape == y.shape
    assert float((yc - y).norm() / y.norm()) < 0.2
    batched = WaveOperatorB200(dom, src, rec, source_batch=2, **kw)
    assert torch.allclose(batched({"c": c}), y, atol=1e-12)
    with pytest.raises(OperatorError, match="exceeds"):
        op({"c": torch.full((32, 32), 3.0, dtype=torch.float64, device=cuda_device)})


def test_energy_is_conserved_without_absorption(cuda_device):
    """tests/test_physics_wave.py:100-118 through the per-step observe path."""
    dom = Domain((40, 40), ((0.0, 1.0), (0.0, 1.0)))
    c = torch.full((40, 40), 1.0, dtype=torch.float64)
    c[20:, :] = 1.5
    c = c.to(cuda_device)
    op = WaveOperatorB200(dom, [[0.5, 0.5]], [[0.2, 0.2]], n_t=150, dt_obs=0.01, f0=8.0, c_max=1.5,
                          order=4, grad_mode="autograd", absorbing="none")
    rec = list(range(80, 1 + 149 * 2, 20))
    from nefi_b200.geometry import stencil_weights

    wc, w1, w2 = stencil_weights(op.grid.spacing, 4)

    def lap(p):  # order-4 Laplacian, zero outside the grid
        out = wc * p
        for ax in (0, 1):
            for o, w in ((1, w1[ax]), (2, w2[ax])):
                out = out + w * (_shift(p, o, -2 + ax) + _shift(p, -o, -2 + ax))
        return out

    def energy(state, n):
        pp, p = state
        kin = (p - pp) ** 2 / (c**2 * op.dt**2)
        return 0.5 * (kin - p * lap(pp)).sum()

    _, e = op.simulate(c, observe=energy, record=rec)
    e = torch.stack(e)
    assert float((e.max() - e.min()) / e.mean()) < 1e-9


def _shift(p, o, dim):
    out = torch.zeros_like(p)
    n = p.shape[dim]
    if o > 0:
        out.narrow(dim, o, n - o).copy_(p.narrow(dim, 0, n - o))
    else:
        out.narrow(dim, 0, n + o).copy_(p.narrow(dim, -o, n + o))
    return out


@pytest.mark.parametrize("snapshot", ["fp16", "delta16"])
def test_corrupted_snapshot_raises(snapshot, cuda_device):
    """Host-side fault injection: a NaN written into the snapshot pool between the forward and the
    backward sweep must surface as SolverError, not as a silent gradient."""
    case = load_golden("fwi_o4_sponge")
    op = make_op(case, grad_mode="checkpoint", checkpoint_every=10, snapshot=snapshot)
    c = torch.tensor(case["c"], dtype=torch.float32, device=cuda_device, requires_grad=True)
    tr = op({"c": c})
    ctx_run = tr.grad_fn.run  # the _Run object saved on the autograd context
    ctx_run.snap.view(torch.float32).fill_(float("nan"))  # poison every block and scale
    with pytest.raises(SolverError, match="non-finite"):
        tr.sum().backward()
    # the context stays usable afterwards
    tr2 = op({"c": c.detach()})
    assert torch.isfinite(tr2).all()


def test_oracle_agrees_with_device_float32_on_cfg1(cuda_device):
    case = load_golden("cfg1_128_o4_sponge")
    tr, gc = run_fwi(case, torch.float32, cuda_device)
    orc = oracle_for(case)
    g = cotangent(full_trace_shape(case), case["seed"])
    otr, ogc = orc.fwi(case["c"], g, dtype=np.float64)
    assert rel_l2(tr, otr[:, :: case["rec_stride"]]) < 1e-5
    assert rel_l2(gc, ogc) < 1e-4


def _layered_op(n=200, shots=6, n_t=81, **kw):
    """A 200^2 (240^2 padded) sponge problem with several shots, so that shot groups, partial
    groups and many tiles (absorbing-layer and interior ones) all occur."""
    h = 10.0
    dom = Domain((n, n), ((0.0, n * h), (0.0, n * h)))
    src = [[(k + 0.5) * n * h / shots, 1.5 * h] for k in range(shots)]
    rec = [[(i + 0.5) * h, 2.5 * h] for i in range(0, n, 3)]
    return WaveOperatorB200(dom, src, rec, n_t=n_t, dt_obs=8e-4, f0=15.0, c_max=3000.0, order=4,
                            absorbing="sponge", absorb_width=20 * h, courant=1.0, grad_mode="autograd", **kw)


def _layered_grad(op, dtype, dev, tuning):
    op.tuning = tuning
    op._plans.clear()
    n = op.grid.shape[0]
    x = torch.linspace(0, 1, n, dtype=torch.float64)
    c = (2000.0 + 800.0 * x[None, :] + 150.0 * torch.sin(7 * x)[:, None]).to(dtype).to(dev)
    c.requires_grad_(True)
    tr = op({"c": c})
    g = torch.randn(tr.shape, generator=torch.Generator().manual_seed(5), dtype=torch.float64).to(dtype).to(dev)
    (gc,) = torch.autograd.grad((tr * g).sum(), c)
    return tr.detach().cpu().numpy(), gc.double().cpu().numpy()


# (vz, rx, shots_per_cta, adj_vz, adj_rx, adj_shots_per_cta)
LAUNCH_SHAPES = [(2, 2, 1, 2, 2, 1), (2, 8, 2, 2, 4, 3), (4, 4, 3, 4, 2, 1), (4, 2, 8, 2, 8, 8)]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_results_do_not_depend_on_the_launch_shape(dtype, cuda_device):
    """Traces are bitwise the same for every tile shape and shot grouping (each cell is computed by
    the same arithmetic); the gradient only regroups its float sums (float64: 1e-12, float32: 1e-5)."""
    op = _layered_op()
    tr0, g0 = _layered_grad(op, dtype, cuda_device, (0, 0, 0, 0, 0, 0))
    assert np.isfinite(g0).all() and np.abs(g0).max() > 0
    for shape in LAUNCH_SHAPES:
        if dtype == torch.float64 and (shape[0] == 4 or shape[3] == 4):
            continue  # float64 tiles are 2 columns per thread
        tr, g = _layered_grad(op, dtype, cuda_device, shape)
        assert np.array_equal(tr, tr0), shape
        assert rel_l2(g, g0) < (1e-12 if dtype == torch.float64 else 1e-5), shape


def test_autotune_chooses_the_launch_shape_and_the_depth(cuda_device):
    """The operator's autotuner times forward shapes with one and two steps per launch and adjoint
    shapes, keeps the fastest, and the chosen tuning gives the default's traces bitwise and its
    gradient up to the regrouped sums."""
    op = _layered_op()
    tr0, g0 = _layered_grad(op, torch.float32, cuda_device, None)
    n = op.grid.shape[0]
    x = torch.linspace(0, 1, n, dtype=torch.float64)
    c = (2000.0 + 800.0 * x[None, :] + 150.0 * torch.sin(7 * x)[:, None]).to(torch.float32).to(cuda_device)
    tu = op.autotune(c, steps=60, repeats=1)
    assert len(tu) == 7 and tu[6] in (1, 2)
    assert any(k[6] == 2 for k in op.autotune_results), "depth 2 is among the timed candidates"
    assert all(f > 0 and a > 0 for f, a in op.autotune_results.values())
    tr, g = _layered_grad(op, torch.float32, cuda_device, tu)
    assert np.array_equal(tr, tr0)
    assert rel_l2(g, g0) < 1e-5


# (vz, rx, shots_per_cta) of the forward with two steps per launch
TWO_STEP_SHAPES = [(4, 2, 2), (4, 4, 2), (2, 4, 3), (4, 8, 1), (2, 2, 8)]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_two_steps_per_launch_are_bitwise_one_step(dtype, cuda_device):
    """The forward taking two leapfrog steps per launch (temporal blocking) gives bitwise the traces and
    the gradient of one step per launch, for every tile shape, with an odd step count (a final single
    step) and on a grid whose tiles straddle the absorbing layer and the grid's edges."""
    op = _layered_op(n=150, shots=5, n_t=62)
    tr1, g1 = _layered_grad(op, dtype, cuda_device, (0, 0, 0, 0, 0, 0, 1))
    assert op.n_steps % 2 == 1
    for vz, rx, spc in TWO_STEP_SHAPES:
        if dtype == torch.float64 and vz == 4:
            continue
        tr2, g2 = _layered_grad(op, dtype, cuda_device, (vz, rx, spc, 0, 0, 0, 2))
        assert op._plan(cuda_device, dtype).ring_levels == 4
        assert np.array_equal(tr2, tr1), (vz, rx, spc)
        assert np.array_equal(g2, g1), (vz, rx, spc)


@pytest.mark.parametrize("name", ["fwi_o4_sponge", "fwi_o2_none", "fwi_o4_cerjan", "fwi_o2_sponge_aniso",
                                  "cfg1_128_o4_sponge"])
def test_two_steps_per_launch_match_the_reference(name, cuda_device):
    """The reference's fixtures through two steps per launch: float64 to rounding, float32 bitwise the
    one-step results, in full-history and checkpointed (binomial, 16-bit) storage."""
    case = load_golden(name)
    tr64, gc64 = run_fwi(case, torch.float64, cuda_device, tuning=(0, 0, 0, 0, 0, 0, 2))
    assert rel_l2(tr64, case["traces_f64"]) < 1e-11
    assert rel_l2(gc64, case["grad_c_f64"]) < 1e-10
    for over in ({}, {"grad_mode": "checkpoint", "checkpoint_every": 7, "checkpoint_slots": 2,
                      "snapshot": "delta16"}):
        one = run_fwi(case, torch.float32, cuda_device, tuning=(0, 0, 0, 0, 0, 0, 1), **over)
        two = run_fwi(case, torch.float32, cuda_device, tuning=(0, 0, 0, 0, 0, 0, 2), **over)
        assert np.array_equal(one[0], two[0]) and np.array_equal(one[1], two[1]), over


def test_two_steps_per_launch_in_the_photoacoustic_operator(cuda_device):
    case = load_golden("pat2d_o4_sponge")
    ref = run_pat(case, torch.float32, cuda_device, tuning=(0, 0, 0, 0, 0, 0, 1), with_c=True)
    got = run_pat(case, torch.float32, cuda_device, tuning=(0, 0, 0, 0, 0, 0, 2), with_c=True)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


def _pml_interior_case():
    """A PML grid whose interior holds several tiles, so the interior runs through the tiled kernels
    and only the layer through the PML kernel (the geometry of the ``fwi_o4_pml_box`` fixture)."""
    g = torch.Generator().manual_seed(21)
    shape, extent = (56, 200), ((0.0, 0.56), (0.0, 2.0))
    c = (2.0 + 0.15 * torch.randn(shape, generator=g, dtype=torch.float64)).clamp(1.7, 2.3)
    c = torch.nn.functional.avg_pool2d(c[None, None], 5, 1, 2, count_include_pad=False)[0, 0]
    src = [[0.05, 0.4], [0.3, 1.5]]
    rec = [[0.02, 0.1 + 0.09 * i] for i in range(20)] + [[0.5, 1.0]]
    kw = dict(n_t=50, dt_obs=0.004, f0=25.0, c_max=2.5, order=4, absorbing="pml", absorb_width=0.08)
    return shape, extent, c, src, rec, kw


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_pml_box_fixture_sends_its_interior_through_the_tiled_kernels(dtype, cuda_device):
    """The reference fixture ``fwi_o4_pml_box`` (checked by the float64/float32 parity tests above)
    has a trivial interior box larger than the forward and the adjoint tiles, after the box's first
    column is rounded up to a 16-byte boundary."""
    case = load_golden("fwi_o4_pml_box")
    plan = make_op(case)._plan(cuda_device, dtype)
    x0, x1, z0, z1 = plan.pml["core"]
    epc = 16 // torch.tensor([], dtype=dtype).element_size()
    z0 = -(-z0 // epc) * epc
    for tx, tz in (plan.tile, plan.adj_tile):
        assert x1 - x0 >= tx and z1 - z0 >= tz


@pytest.mark.parametrize("dtype,tt,tg", [(torch.float64, 1e-11, 1e-10), (torch.float32, 1e-5, 1e-4)])
def test_pml_interior_through_tiled_kernels_matches_the_oracle(dtype, tt, tg, cuda_device):
    import oracle

    shape, extent, c, src, rec, kw = _pml_interior_case()
    dom = Domain(shape, extent)
    op = WaveOperatorB200(dom, src, rec, grad_mode="autograd", **kw)
    x0, x1, z0, z1 = op._plan(cuda_device, dtype).pml["core"]
    assert x1 - x0 >= 32 and z1 - z0 >= 128  # larger than the default forward and adjoint tiles
    # every receiver-touched cell lies in the tiled box: the box's adjoint launch adds the cotangents
    assert op._plan(cuda_device, dtype).adj_tables_box == 1
    cd = c.to(dtype).to(cuda_device).requires_grad_(True)
    tr = op({"c": cd})
    gt = torch.tensor(cotangent(tr.shape, 22), dtype=dtype, device=cuda_device)
    (gc,) = torch.autograd.grad((tr * gt).sum(), cd)
    orc = oracle.OracleWave(shape, extent, np.asarray(rec), sources=np.asarray(src), **kw)
    tr_o, gc_o = orc.fwi(c.numpy(), cotangent(tr.shape, 22), dtype=np.float64)
    assert rel_l2(tr.detach().cpu().numpy(), tr_o) < tt
    assert rel_l2(gc.cpu().numpy(), gc_o) < tg
    # checkpointed (exact snapshots): bitwise the same gradient
    opk = WaveOperatorB200(dom, src, rec, grad_mode="checkpoint", checkpoint_every=9, **kw)
    cd2 = c.to(dtype).to(cuda_device).requires_grad_(True)
    (gk,) = torch.autograd.grad((opk({"c": cd2}) * gt).sum(), cd2)
    assert torch.equal(gk, gc)


@pytest.mark.parametrize("dtype,tt,tg", [(torch.float64, 1e-11, 1e-10), (torch.float32, 1e-5, 1e-4)])
def test_pml_cotangents_of_layer_cells_match_the_oracle(dtype, tt, tg, cuda_device):
    """Receivers on the domain's faces reach the first layer row and column: the box's adjoint launch
    adds the cotangents of the touched cells inside the tiled box and the layer launch those of the
    listed cells outside it; traces and gradient against the float64 oracle, and checkpointed
    (exact snapshots) bitwise the history gradient."""
    import oracle

    shape, extent, c, src, rec, kw = _pml_interior_case()
    rec = rec + [[0.0, 0.77], [0.33, 0.0], [0.56, 1.3], [0.41, 2.0]]  # on the four faces
    dom = Domain(shape, extent)
    op = WaveOperatorB200(dom, src, rec, grad_mode="autograd", **kw)
    plan = op._plan(cuda_device, dtype)
    assert plan.adj_tables_box == 1 and plan.layer_cell_index.numel() > 0
    cd = c.to(dtype).to(cuda_device).requires_grad_(True)
    tr = op({"c": cd})
    gt = torch.tensor(cotangent(tr.shape, 23), dtype=dtype, device=cuda_device)
    (gc,) = torch.autograd.grad((tr * gt).sum(), cd)
    orc = oracle.OracleWave(shape, extent, np.asarray(rec), sources=np.asarray(src), **kw)
    tr_o, gc_o = orc.fwi(c.numpy(), cotangent(tr.shape, 23), dtype=np.float64)
    assert rel_l2(tr.detach().cpu().numpy(), tr_o) < tt
    assert rel_l2(gc.cpu().numpy(), gc_o) < tg
    opk = WaveOperatorB200(dom, src, rec, grad_mode="checkpoint", checkpoint_every=7, **kw)
    cd2 = c.to(dtype).to(cuda_device).requires_grad_(True)
    (gk,) = torch.autograd.grad((opk({"c": cd2}) * gt).sum(), cd2)
    assert torch.equal(gk, gc)


def test_pml_forward_captured_in_a_fresh_thread(cuda_device):
    """A PML forward sweep (its layer kernel on the calling thread's second stream) captured into a
    CUDA graph by a thread that never ran one: the second stream is created inside the capture, and
    the replay equals the eager sweep."""
    import ctypes as C
    import threading

    from nefi_b200 import _lib
    from nefi_b200.operators import _forward_sweep, _Run

    shape, extent, c, src, rec, kw = _pml_interior_case()
    op = WaveOperatorB200(Domain(shape, extent), src, rec, grad_mode="autograd", **kw)
    plan = op._plan(cuda_device, torch.float32)
    S = op.n_sources
    cd = c.float().to(cuda_device).contiguous()
    c2dt2 = torch.empty(plan.field, device=cuda_device, dtype=torch.float32)
    _lib.check(_lib.load().nw_prepare_medium(C.byref(plan.g), plan.n_abs, cd.data_ptr(), op.dt**2,
                                             c2dt2.data_ptr(), _lib.stream_handle(cuda_device)))
    medium, acq = plan.medium(c2dt2), plan.acquisition(S)
    run = _Run(plan, S, op.n_steps, ("ring", None), "exact")
    traces = torch.zeros(S, plan.n_rec, op.n_t, device=cuda_device)

    def sweep(stream_handle):
        run.ring.zero_()
        run.psi.zero_()
        _forward_sweep(plan, medium, acq, run, 0, op.n_steps, traces, stream_handle)

    sweep(_lib.stream_handle(cuda_device))  # this thread: kernels loaded, shared-memory opt-ins done
    torch.cuda.synchronize(cuda_device)
    eager = traces.clone()
    traces.zero_()
    out = {}

    def worker():
        try:
            torch.cuda.set_device(cuda_device)
            st = torch.cuda.Stream(cuda_device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(st):
                with torch.cuda.graph(g, stream=st):
                    sweep(st.cuda_stream)
            g.replay()
            torch.cuda.synchronize(cuda_device)
            out["y"] = traces.clone()
        except Exception as e:  # reported by the main thread
            out["err"] = e

    t = threading.Thread(target=worker)
    t.start()
    t.join(timeout=300)
    assert "err" not in out, out.get("err")
    assert torch.equal(out["y"], eager)


@pytest.mark.parametrize("seed", range(8))
@pytest.mark.parametrize("dtype,tt,tg", [(torch.float64, 1e-11, 1e-10), (torch.float32, 1e-5, 1e-4)])
def test_random_geometries_match_the_oracle_and_the_reference(seed, dtype, tt, tg, cuda_device):
    """Seeded random 2-D geometries (tests/random_geometry.py: grid shape and spacing, every layer
    kind, order, substeps, several shots, receivers anywhere, long enough for the wave to cross the
    domain) through the device path: traces and the gradient of ``sum(traces * g)`` against the
    float64 oracle, and in float32 also against the reference's own float32 and float64 runs of the
    same problems (tests/golden/random/random_<seed>.npz, written by make_random_golden.py)."""
    import oracle
    from random_geometry import random_geometry

    p = random_geometry(seed)
    (n0, n1), ext, src, rec, kw, c, gt = p["shape"], p["extent"], p["sources"], p["receivers"], p["kw"], p["c"], p["gt"]
    op = WaveOperatorB200(Domain((n0, n1), ext), src, rec, grad_mode="autograd", **kw)
    cd = torch.tensor(c, dtype=dtype, device=cuda_device).requires_grad_(True)
    tr = op({"c": cd})
    (gc,) = torch.autograd.grad((tr * torch.tensor(gt, dtype=dtype, device=cuda_device)).sum(), cd)
    tr, gc = tr.detach().cpu().numpy(), gc.cpu().numpy()
    orc = oracle.OracleWave((n0, n1), ext, np.asarray(rec), sources=np.asarray(src), **kw)
    tr_o, gc_o = orc.fwi(c, gt, dtype=np.float64)
    assert np.linalg.norm(tr_o) > 0 and np.linalg.norm(gc_o) > 0  # the wave reaches the receivers
    ref = np.load(Path(__file__).parent / "golden" / "random" / f"random_{seed}.npz")
    if dtype == torch.float32:
        # float32 rounding grows with the step count (up to 1200 steps here): the bound is twice the
        # reference's own float32 error against its float64 run of the same problem
        r_tr, r_gc = rel_l2(ref["traces_f32"], ref["traces_f64"]), rel_l2(ref["grad_f32"], ref["grad_f64"])
        tt, tg = max(tt, 2.0 * r_tr), max(tg, 2.0 * r_gc)
        # a fixed ceiling, so that a drifting reference error cannot hide a device regression
        assert tt <= 1e-4 and tg <= 1e-3, (tt, tg)
        d_tr, d_gc = rel_l2(tr, ref["traces_f64"]), rel_l2(gc, ref["grad_f64"])
        v_tr, v_gc = rel_l2(tr, ref["traces_f32"]), rel_l2(gc, ref["grad_f32"])
        print(f"seed {seed} {kw['absorbing']}: device float32 vs reference float64 traces {d_tr:.2e}, gradient "
              f"{d_gc:.2e}; vs reference float32 {v_tr:.2e}, {v_gc:.2e}; reference float32 vs float64 "
              f"{r_tr:.2e}, {r_gc:.2e}")
        assert d_tr < tt and d_gc < tg, (kw, d_tr, d_gc)
        assert v_tr < tt and v_gc < tg, (kw, v_tr, v_gc)
    else:  # the fixtures are stored in float32: agreement to their rounding
        assert rel_l2(tr, ref["traces_f64"]) < 1e-6 and rel_l2(gc, ref["grad_f64"]) < 1e-6
    e_tr, e_gc = rel_l2(tr, tr_o), rel_l2(gc, gc_o)
    print(f"seed {seed} {kw['absorbing']} {dtype}: vs the float64 oracle traces {e_tr:.2e} (bound {tt:.1e}), "
          f"gradient {e_gc:.2e} (bound {tg:.1e})")
    assert e_tr < tt, (kw["absorbing"], kw)
    assert e_gc < tg, (kw["absorbing"], kw)


def test_pat_float64_matches_the_oracle_on_a_96_cube(cuda_device):
    """The float64 3-D photoacoustic path that the large 3-D configuration's accuracy figure is measured
    against, checked against the float64 oracle at 96^3 (10-cell sponge, order 2, two instances, a
    sensor plane on one face, 120 steps): traces, and the gradients w.r.t. p0 and c."""
    import oracle
    from nefi_b200.workloads import pat_volume

    w = pat_volume(n=96, batch=2, n_steps=120, seed=1, n_sensors=24)
    kw = {**w.operator_kwargs(), "absorb_width": 10 * w.h}
    op = WaveInitialConditionOperatorB200(w.domain, w.sensors, grad_mode="checkpoint", **kw)
    p0 = torch.tensor(w.p0, dtype=torch.float64, device=cuda_device, requires_grad=True)
    c = torch.tensor(w.c, dtype=torch.float64, device=cuda_device, requires_grad=True)
    tr = op.with_speed(p0, c)
    g = np.random.default_rng(3).standard_normal(tuple(tr.shape))
    gp, gc = torch.autograd.grad((tr * torch.tensor(g, device=cuda_device)).sum(), (p0, c))
    okw = {k: v for k, v in kw.items() if k != "c"}
    orc = oracle.OracleWave(w.domain.shape, w.domain.extent, w.sensors, c_max=float(w.c.max()), **okw)
    oracle.set_threads(max(1, __import__("os").cpu_count() or 1))
    otr, ogp, ogc = orc.pat(w.p0, w.c, g, dtype=np.float64)
    assert rel_l2(tr.detach().cpu().numpy(), otr) < 1e-11
    assert rel_l2(gp.cpu().numpy(), ogp) < 1e-10
    assert rel_l2(gc.cpu().numpy(), ogc) < 1e-10
