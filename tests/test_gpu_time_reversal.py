"""GPU parity of the classical PAT baseline ``time_reversal`` (nefi/physics/wave.py:878-968).

``mode="dirichlet"`` runs on the device through ``nw_time_reversal`` and is compared with the
reference's own output on the committed fixtures (relative L2: float64 1e-11, float32 1e-5).
``mode="adjoint"`` is the exact adjoint of the photoacoustic operator: with the fixtures' cotangent
as traces it reproduces the reference's ``d<traces, g>/dp0`` (float64 1e-10, float32 1e-4).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import cotangent, golden_names, load_golden, rel_l2
from nefi_b200 import time_reversal
from nefi_b200._compat import ConfigError, Domain, ShapeError

pytestmark = pytest.mark.gpu

TR_KW = ("order", "absorbing", "absorb_width", "absorb_R", "courant")


def _domain(case):
    return Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))


@pytest.mark.parametrize("name", golden_names("tr"))
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 1e-5)])
def test_dirichlet_time_reversal_matches_reference(name, dtype, tol):
    case = load_golden(name)
    kw = {k: v for k, v in case["kw"].items() if k in TR_KW}
    tr = torch.tensor(case["traces"], dtype=dtype, device="cuda")
    p0 = time_reversal(tr, _domain(case), case["receivers"], dt_obs=case["kw"]["dt_obs"],
                       c=torch.tensor(case["c"]), mode="dirichlet", **kw)
    assert p0.dtype == dtype and p0.device.type == "cuda" and tuple(p0.shape) == tuple(case["shape"])
    ref = case["p0_f64"] if dtype == torch.float64 else case["p0_f32"]
    assert rel_l2(p0.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("name", golden_names("pat"))
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-10), (torch.float32, 1e-4)])
def test_adjoint_time_reversal_is_the_operator_adjoint(name, dtype, tol):
    case = load_golden(name)
    kw = {k: v for k, v in case["kw"].items() if k in TR_KW}
    shape = (len(case["receivers"]), case["kw"]["n_t"])
    g = torch.tensor(cotangent((1, *shape), case["seed"]), dtype=dtype, device="cuda")
    p0 = time_reversal(g, _domain(case), case["receivers"], dt_obs=case["kw"]["dt_obs"],
                       c=torch.tensor(case["c"]), mode="adjoint", **kw)
    ref = case["grad_p0_f64"] if dtype == torch.float64 else case["grad_p0_f32"]
    # a batched fixture's first image: its cotangent is the first (n_receivers, n_t) of the draw
    ref = ref.reshape(-1, *p0.shape)[0]
    assert rel_l2(p0.detach().cpu().numpy(), ref) < tol


def test_time_reversal_argument_errors():
    case = load_golden(golden_names("tr")[0])
    dom = _domain(case)
    tr = torch.tensor(case["traces"], dtype=torch.float32, device="cuda")
    with pytest.raises(ConfigError):
        time_reversal(tr, dom, case["receivers"], dt_obs=0.03, mode="forward")
    with pytest.raises(ShapeError):
        time_reversal(tr[None, None], dom, case["receivers"], dt_obs=0.03)
    with pytest.raises(ShapeError):
        time_reversal(tr[:-1], dom, case["receivers"], dt_obs=0.03)


def test_coincident_receivers_keep_the_last_trace():
    """Two receivers in one cell: the later one's trace holds the cell (the reference assigns the
    cells in receiver order)."""
    case = load_golden("tr2d_o2_sponge")
    dom = _domain(case)
    kw = {k: v for k, v in case["kw"].items() if k in TR_KW}
    rec = np.concatenate([case["receivers"], case["receivers"][:1]])
    tr = torch.tensor(case["traces"], dtype=torch.float64, device="cuda")
    tr2 = torch.cat([tr, 0.5 * tr[:1]])
    a = time_reversal(tr2, dom, rec, dt_obs=case["kw"]["dt_obs"], c=1.0, **kw)
    rec_b, tr_b = rec[1:], tr2[1:]
    b = time_reversal(tr_b, dom, rec_b, dt_obs=case["kw"]["dt_obs"], c=1.0, **kw)
    assert torch.equal(a, b)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_initial_condition_operator_is_linear_and_time_reversal_refocuses(dtype):
    """tests/test_physics_wave.py:192-214 on the device: the photoacoustic operator is linear, and
    both reversal modes put the image's peak within 3 cells of a Gaussian source, correlated with
    it above 0.5."""
    import math

    from nefi_b200 import WaveInitialConditionOperatorB200

    n = 48
    dom = Domain((n, n), ((-1.0, 1.0), (-1.0, 1.0)))
    th = 2 * math.pi * torch.arange(64, dtype=torch.float64) / 64
    rec = torch.stack([0.9 * torch.cos(th), 0.9 * torch.sin(th)], 1)
    op = WaveInitialConditionOperatorB200(dom, rec, n_t=200, dt_obs=0.01, c=1.0, absorb_width=0.25)
    assert op.homogeneity == 1.0
    x = dom.physical_coords(dtype=torch.float64)
    src = torch.tensor([0.3, -0.2], dtype=torch.float64)
    p0 = torch.exp(-((x - src) ** 2).sum(-1) / (2 * 0.05**2)).to("cuda", dtype)
    q0 = torch.randn(n, n, dtype=torch.float64, generator=torch.Generator().manual_seed(0)).to("cuda", dtype)
    y1, y2 = op({"p0": p0}), op({"p0": q0})
    y3 = op({"p0": 2 * p0 - 3 * q0})
    assert y1.shape == (64, 200)
    lin = float((y3 - (2 * y1 - 3 * y2)).norm() / y3.norm())
    assert lin < (1e-10 if dtype == torch.float64 else 1e-5)
    for mode in ("dirichlet", "adjoint"):
        img = time_reversal(y1, dom, rec, dt_obs=0.01, c=1.0, mode=mode)
        assert img.dtype == dtype and tuple(img.shape) == (n, n)
        i = int(torch.argmax(img))
        peak = x.reshape(-1, 2)[i]
        assert float((peak - src).norm()) < 3 * dom.spacing()[0], (mode, peak)
        corr = torch.corrcoef(torch.stack([img.flatten().double(), p0.flatten().double()]))[0, 1]
        assert float(corr) > 0.5, (mode, float(corr))
