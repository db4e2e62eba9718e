"""FP64 data generation on the device, the way ``DataGenerator.clean`` drives an operator
(nefi/bench/base.py:74-90): the operator is moved to float64 and the device, then called through
``at_resolution`` with the ground truth on a 2x-refined grid (the wave_fwi generator,
nefi/instances/wave_fwi/__init__.py:248-260). The traces must equal the reference's float64 traces
to rounding (relative L2 1e-11)."""

from __future__ import annotations

import pytest
import torch

from conftest import golden_names, load_golden, rel_l2
from nefi_b200 import WaveOperatorB200
from nefi_b200._compat import Domain

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_names("gen"))
def test_fp64_supersampled_generation_matches_reference(name, cuda_device):
    case = load_golden(name)
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    op = WaveOperatorB200(dom, case["sources"], case["receivers"], **case["kw"])
    op = op.to(device=cuda_device, dtype=torch.float64)
    fields = {"c": torch.as_tensor(case["c"]).to(cuda_device, torch.float64)}
    with torch.no_grad():
        fine = op.at_resolution(tuple(case["fine"]))
        tr = fine(fields)
    assert fine is op.at_resolution(tuple(case["fine"])) and fine.grid.shape == tuple(case["fine"])
    assert tr.dtype == torch.float64 and tr.device.type == "cuda"
    assert rel_l2(tr.cpu().numpy(), case["traces_f64"]) < 1e-11


def test_photoacoustic_at_resolution_resamples_the_speed_like_the_reference(cuda_device):
    """The photoacoustic operator at a finer resolution resamples its known speed map before the run
    (nefi/physics/wave.py:822-835): float64 traces equal the reference's to rounding."""
    from nefi_b200 import WaveInitialConditionOperatorB200

    case = load_golden("genpat2x_o4_sponge")
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    op = WaveInitialConditionOperatorB200(dom, case["receivers"], c=torch.tensor(case["c"]), **case["kw"])
    fine = op.to(device=cuda_device, dtype=torch.float64).at_resolution(tuple(case["fine"]))
    with torch.no_grad():
        tr = fine({"p0": torch.tensor(case["p0"], dtype=torch.float64, device=cuda_device)})
    assert rel_l2(tr.cpu().numpy(), case["traces_f64"]) < 1e-11
