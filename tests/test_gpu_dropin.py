"""The drop-in inside NEFI itself, on the GPU: NEFI's own instances and property checks with the wave
operator classes swapped for the B200 ones, the base class being the real
``nefi.operators.base.Operator``.

These tests need the ``nefi`` package importable (``tests/conftest.py`` puts an installed copy on
``sys.path`` when one is present) and are skipped otherwise. They restate, with the operator swapped
and on ``cuda``, the reference's checks:

* ``tests/test_instances_wave_family.py:58-62`` (``test_wave_fwi_smoke``): ``WaveFWI(steps=(20, 30))``
  runs its whole curriculum through ``Solver._run_stage`` (nefi/solve/solver.py:349,427), which calls
  the operator as ``op(fields)`` and back-propagates through it, after generating its data in
  float64 on a 2x finer grid (``DataGenerator.clean``, nefi/bench/base.py:86-90, pointed at the GPU);
  the data loss must fall below half its start and the recovered speed must beat the initial guess
  (``_check_common``, :22-36);
* ``tests/test_physics_wave.py:145-165``: checkpointed and full-history gradients agree, and agree
  with central finite differences, in float64;
* ``tests/test_photoacoustic3d.py:49-59``: linearity and the exact adjoint identity of the
  photoacoustic operator behind ``SensorBandwidth``, in float64.
"""

from __future__ import annotations

import pytest
import torch

from nefi_b200 import WaveInitialConditionOperatorB200, WaveOperatorB200
from nefi_b200 import _compat

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not _compat.HAVE_NEFI, reason="the nefi package is not importable")]

F64 = torch.float64


def test_the_b200_operators_subclass_nefis_operator():
    from nefi.operators.base import Operator
    from nefi.registry import build

    assert issubclass(WaveOperatorB200, Operator) and issubclass(WaveInitialConditionOperatorB200, Operator)
    dom = _compat.Domain((16, 16), ((0.0, 1.0), (0.0, 1.0)))
    op = build("operator", {"type": "wave_b200", "domain": dom, "sources": [[0.2, 0.3]],
                            "receivers": [[0.8, 0.5]], "n_t": 10, "dt_obs": 0.01, "f0": 5.0, "c_max": 2.5})
    assert isinstance(op, WaveOperatorB200)


def test_wave_fwi_instance_runs_on_the_b200_operator(cuda_device, monkeypatch):
    import nefi.instances.wave_fwi as wf
    from nefi.instances.wave_fwi import WaveFWI
    from nefi.metrics import evaluate

    monkeypatch.setattr(wf, "WaveOperator", WaveOperatorB200)
    # NEFI's data generator simulates on the CPU unless told otherwise (nefi/bench/base.py:68-80); the
    # B200 operator has no CPU path, so the instance's float64 data generation is pointed at the GPU
    gen_init = wf.TraceDataGenerator.__init__

    def gen_on_device(self, operator, trace_mask=None, **kw):
        kw.setdefault("device", cuda_device)
        gen_init(self, operator, trace_mask=trace_mask, **kw)

    monkeypatch.setattr(wf.TraceDataGenerator, "__init__", gen_on_device)
    inst = WaveFWI(steps=(20, 30))
    assert isinstance(inst.operator(), WaveOperatorB200)
    out = inst.run(seed=0, device=str(cuda_device))
    res, gt, meas = out.result, out.gt, out.measurement
    n = inst.cfg.n
    assert res.fields["c"].shape == (n, n)
    assert tuple(res.pred.shape) == tuple(meas.data.shape)
    h = res.history
    data = h["data_loss"] if "data_loss" in h else h["data"]
    assert data[-1] < 0.5 * data[0], (data[0], data[-1])
    init = evaluate(torch.full((n, n), inst.cfg.c_background), gt["c"].cpu(), inst.metrics())
    assert out.metrics["psnr"] > init["psnr"], (out.metrics, init)
    assert out.metrics["anomaly_error"] < init["anomaly_error"]
    problem = inst.build_problem(meas)
    assert isinstance(problem.operator, WaveOperatorB200)
    assert inst.data_generator().fidelity_tag != problem.operator.fidelity_tag


def test_checkpoint_gradients_equal_autograd_and_finite_differences(cuda_device):
    torch.manual_seed(0)
    dom = _compat.Domain((16, 16), ((0.0, 1.0), (0.0, 1.0)))
    c = (2.0 + 0.2 * torch.randn(16, 16, dtype=F64)).clamp(1.6, 2.4).to(cuda_device)
    kw = dict(n_t=40, dt_obs=0.01, f0=5.0, c_max=2.5, absorb_width=0.2)
    src, rec = [[0.2, 0.3], [0.2, 0.7]], [[0.8, y] for y in (0.2, 0.4, 0.6, 0.8)]
    w = torch.randn(2, 4, 40, dtype=F64).to(cuda_device)
    grads = []
    for mode, ck in (("autograd", None), ("checkpoint", 5), ("checkpoint", None)):
        op = WaveOperatorB200(dom, src, rec, grad_mode=mode, checkpoint_every=ck, **kw)
        x = c.clone().requires_grad_(True)
        (g,) = torch.autograd.grad((op({"c": x}) * w).sum(), x)
        grads.append(g)
    for g in grads[1:]:
        assert float((g - grads[0]).norm() / grads[0].norm()) < 1e-6
    op = WaveOperatorB200(dom, src, rec, grad_mode="autograd", **kw)
    e = torch.randn(16, 16, dtype=F64).to(cuda_device)
    eps = 1e-6
    fd = float((op({"c": c + eps * e}) * w).sum()) - float((op({"c": c - eps * e}) * w).sum())
    fd /= 2 * eps
    assert abs(fd - float((grads[0] * e).sum())) < 1e-6 * max(1.0, abs(fd))


def test_photoacoustic_linearity_and_exact_adjoint(cuda_device, monkeypatch):
    import nefi.instances.photoacoustic3d as pa
    from nefi.instances.photoacoustic3d import Photoacoustic3D

    monkeypatch.setattr(pa, "WaveInitialConditionOperator", WaveInitialConditionOperatorB200)
    inst = Photoacoustic3D(extent=(3.0, 3.0, 2.0), grid=(12, 12, 8), t_max=3.0, sensor_grid=(4, 4))
    op = inst.operator().to(F64)
    assert isinstance(op.inner, WaveInitialConditionOperatorB200)
    torch.manual_seed(0)
    a = torch.rand(12, 12, 8, dtype=F64).to(cuda_device)
    b = torch.rand(12, 12, 8, dtype=F64).to(cuda_device)
    ya, yb = op({"p0": a}), op({"p0": b})
    assert torch.allclose(op({"p0": 2 * a - 0.5 * b}), 2 * ya - 0.5 * yb, atol=1e-10)
    y = torch.randn_like(ya)
    x = torch.zeros(12, 12, 8, dtype=F64, device=cuda_device, requires_grad=True)
    (adj,) = torch.autograd.grad((op({"p0": x}) * y).sum(), x)
    assert float((ya * y).sum()) == pytest.approx(float((a * adj).sum()), rel=1e-9)
