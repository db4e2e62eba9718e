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
