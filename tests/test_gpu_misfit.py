"""GPU parity of the fused trace misfit (``nw_misfit_prepare`` / ``nw_misfit`` / ``nw_trace_filter``)
against the reference's ``BandLimitedMSE``, ``lowpass``, ``gaussian_lowpass`` and ``MSE`` (committed
fixtures) and against the numpy misfit oracle at sizes the fixtures do not reach.

Tolerances (relative): float64 loss 1e-11, filtered traces and gradients 1e-10; float32 loss and
filtered traces 1e-5, gradients 1e-4 (against the reference's float32 results).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden_names, load_golden, rel_l2
from nefi_b200 import _lib
from nefi_b200.misfit import (BandLimitedMSEB200, SensorBandwidthB200, TraceMisfit, band_limited_mse,
                              gaussian_lowpass, lowpass)

pytestmark = pytest.mark.gpu

TOL = {torch.float64: (1e-11, 1e-10), torch.float32: (1e-5, 1e-4)}
TAG = {torch.float64: "f64", torch.float32: "f32"}
DTYPES = [torch.float64, torch.float32]


def _t(x, dtype):
    return torch.as_tensor(np.asarray(x)).to("cuda", dtype)


def _rel(a, b):
    a, b = float(torch.as_tensor(a).detach()), float(b)
    return abs(a - b) / max(abs(b), 1e-300)


class _Meas:
    def __init__(self, data, mask=None):
        self.data, self.mask = data, mask


class _Ctx:
    def __init__(self, pred, obs):
        self.pred, self.obs = pred, obs


@pytest.mark.parametrize("name", golden_names("misfit"))
@pytest.mark.parametrize("dtype", DTYPES)
def test_band_limited_mse_matches_reference(name, dtype):
    case = load_golden(name)
    kw, tag = case["kw"], TAG[dtype]
    tl, tg = TOL[dtype]
    pred = _t(case["pred"], dtype).requires_grad_(True)
    obs = _t(case["obs"], dtype)
    mask = None if "mask" not in case else _t(case["mask"], dtype)
    loss = BandLimitedMSEB200(kw["f_max"], kw["dt"], kw.get("taper", 0.3), kw["relative"]).forward(
        _Ctx(pred, _Meas(obs, mask)))
    (g,) = torch.autograd.grad(loss, pred)
    assert loss.dtype == dtype and loss.ndim == 0
    assert _rel(loss, case[f"loss_{tag}"]) < tl
    assert rel_l2(g.cpu().numpy(), case[f"grad_{tag}"]) < tg
    if kw["f_max"] is not None:
        y = lowpass(pred.detach(), kw["dt"], kw["f_max"], kw.get("taper", 0.3))
        assert rel_l2(y.cpu().numpy(), case[f"lowpass_{tag}"]) < tl


@pytest.mark.parametrize("name", [n for n in golden_names("misfit") if load_golden(n)["sensor"] is not None])
@pytest.mark.parametrize("dtype", DTYPES)
def test_sensor_response_and_its_misfit_match_reference(name, dtype):
    case = load_golden(name)
    tag, (tl, tg) = TAG[dtype], TOL[dtype]
    pred = _t(case["pred"], dtype).requires_grad_(True)
    obs = _t(case["obs"], dtype)
    mask = None if "mask" not in case else _t(case["mask"], dtype)
    y = gaussian_lowpass(pred, case["dt"], case["sensor"])
    assert rel_l2(y.detach().cpu().numpy(), case[f"sensor_{tag}"]) < tl
    mf = TraceMisfit(case["dt"], None, relative=False, sensor_cutoff=case["sensor"])
    mf.prepare(obs, mask)
    loss, g = mf.value_and_grad(pred.detach())
    assert _rel(loss, case[f"sensor_loss_{tag}"]) < tl
    assert rel_l2(g.cpu().numpy(), case[f"sensor_grad_{tag}"]) < tg
    # the same gradient through autograd of the filter (its backward is the same filter)
    m = 1.0 if mask is None else mask
    lo = ((y - obs) ** 2 * m).sum() / (torch.ones_like(obs) * m).sum()
    (ga,) = torch.autograd.grad(lo, pred)
    assert rel_l2(ga.cpu().numpy(), case[f"sensor_grad_{tag}"]) < tg


class _Inner(torch.nn.Module):
    primary, homogeneity = "x", 1.0

    def forward(self, fields):
        return fields["x"] * 2.0

    def at_resolution(self, shape):
        return self

    def output_shape(self, shape):
        return None

    def required_fields(self):
        return ("x",)


def test_sensor_bandwidth_operator_wraps_the_inner_operator():
    case = load_golden("misfit_bl_abs")
    x = _t(case["pred"], torch.float64) * 0.5
    op = SensorBandwidthB200(_Inner(), case["dt"], case["sensor"])
    y = op({"x": x})
    assert rel_l2(y.cpu().numpy(), case["sensor_f64"]) < 1e-10
    assert op.at_resolution((3, 3)) is op and op.required_fields() == ("x",)


@pytest.mark.parametrize("dtype", DTYPES)
def test_large_traces_against_the_oracle(dtype):
    """8001-sample traces (float32, the longest 2^14 filter) and 4001 (float64, 2^13), an odd trace
    count, a per-sample mask, relative and sensor-filtered, against the float64 oracle."""
    import misfit_oracle as mo

    n_t = 8001 if dtype == torch.float32 else 4001
    rng = np.random.default_rng(7)
    t = np.arange(n_t) * 5e-4
    obs = np.sin(2 * np.pi * 30.0 * t)[None, :] * rng.uniform(0.5, 1.5, (37, 1)) + 0.2 * rng.standard_normal((37, n_t))
    pred = obs + 0.3 * rng.standard_normal((37, n_t))
    mask = (rng.uniform(size=(37, n_t)) > 0.1).astype(np.float64)
    lo, go = mo.band_limited_mse(pred, obs, 5e-4, 60.0, 0.3, True, mask, sensor=90.0)
    mf = TraceMisfit(5e-4, 60.0, 0.3, True, sensor_cutoff=90.0)
    mf.prepare(_t(obs, dtype), _t(mask, dtype))
    loss, g = mf.value_and_grad(_t(pred, dtype))
    tl, tg = TOL[dtype]
    assert _rel(loss, lo) < max(tl, 1e-10)
    assert rel_l2(g.cpu().numpy(), go) < tg
    # the same again: the partial sums reduce in a fixed order, so results are bitwise equal
    mf.prepare(_t(obs, dtype), _t(mask, dtype))
    loss2, g2 = mf.value_and_grad(_t(pred, dtype))
    assert float(loss2) == float(loss)
    assert torch.equal(g, g2)


def test_row_slices_accumulate_to_the_whole():
    case = load_golden("misfit_bl_mask")
    kw = case["kw"]
    pred, obs, mask = (_t(case[k], torch.float64) for k in ("pred", "obs", "mask"))
    whole = band_limited_mse(pred, obs, kw["dt"], kw["f_max"], kw["taper"], True, mask)
    mf = TraceMisfit(kw["dt"], kw["f_max"], kw["taper"], True)
    mf.prepare(obs, mask)
    grads = []
    for rows in (slice(0, 3), slice(3, 7)):
        loss, g = mf.value_and_grad(pred[rows], rows=rows)
        grads.append(g)
    assert _rel(loss, whole) < 1e-13
    assert rel_l2(torch.cat(grads).cpu().numpy(), case["grad_f64"]) < 1e-10
    # strided selections (every other row) are gathered, then accumulate the same way
    mf.prepare(obs, mask, always=True)
    g = torch.empty_like(pred)
    for rows in (slice(0, None, 2), slice(1, None, 2)):
        loss, g[rows] = mf.value_and_grad(pred[rows], rows=rows)
    assert _rel(loss, whole) < 1e-13
    assert rel_l2(g.cpu().numpy(), case["grad_f64"]) < 1e-10


def test_filtered_length_limit_is_reported():
    mf = TraceMisfit(1e-3, 50.0)
    with pytest.raises(_lib.LibraryError):
        mf.prepare(torch.zeros(2, 8193, device="cuda"))
    with pytest.raises(_lib.LibraryError):
        lowpass(torch.zeros(2, 4097, device="cuda", dtype=torch.float64), 1e-3, 50.0)


def test_fwi_gradient_with_the_fused_misfit_matches_the_oracle():
    """misfit_gradient(c, d, misfit=TraceMisfit(...)): the band-limited relative misfit's adjoint source
    drives the adjoint sweep; checked against the oracle chain (float64 forward, numpy misfit,
    float64 adjoint) on a reference geometry."""
    import misfit_oracle as mo

    from conftest import oracle_for
    from nefi_b200 import WaveOperatorB200
    from nefi_b200._compat import Domain

    case = load_golden("fwi_o4_sponge")
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    op = WaveOperatorB200(dom, case["sources"], case["receivers"], **case["kw"])
    c = torch.tensor(case["c"], dtype=torch.float64, device="cuda")
    obs = torch.tensor(case["traces_f64"], dtype=torch.float64, device="cuda") * 0.8
    dt_obs = case["kw"]["dt_obs"]
    mf = TraceMisfit(dt_obs, 20.0, 0.3, True)
    loss, grad = op.misfit_gradient(c, obs, misfit=mf)
    orc = oracle_for(case)
    tr, _ = orc.fwi(case["c"], np.zeros(case["traces_f64"].shape), dtype=np.float64)
    lo, gtr = mo.band_limited_mse(tr, obs.cpu().numpy(), dt_obs, 20.0, 0.3, True)
    _, gc = orc.fwi(case["c"], gtr, dtype=np.float64)
    assert _rel(loss, lo) < 1e-10
    assert rel_l2(grad.cpu().numpy(), gc) < 1e-9


def test_fused_misfit_gradient_with_source_chunks_and_a_trace_mute():
    """Shot chunks (source_batch) and a per-trace mask go through the same fused misfit: the loss
    and the gradient equal the unchunked run up to summation order."""
    from nefi_b200 import WaveOperatorB200
    from nefi_b200._compat import Domain

    case = load_golden("fwi_o4_sponge")
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    c = torch.tensor(case["c"], dtype=torch.float64, device="cuda")
    obs = torch.tensor(case["traces_f64"], dtype=torch.float64, device="cuda") * 0.8
    mask = torch.ones(obs.shape[0], obs.shape[1], 1, dtype=torch.float64, device="cuda")
    mask[0, 1] = 0.0
    dt_obs = case["kw"]["dt_obs"]
    whole = WaveOperatorB200(dom, case["sources"], case["receivers"], **case["kw"])
    chunked = WaveOperatorB200(dom, case["sources"], case["receivers"], source_batch=1, **case["kw"])
    l1, g1 = whole.misfit_gradient(c, obs, misfit=TraceMisfit(dt_obs, 20.0), mask=mask)
    l2, g2 = chunked.misfit_gradient(c, obs, misfit=TraceMisfit(dt_obs, 20.0), mask=mask)
    assert _rel(l2, l1) < 1e-12
    assert rel_l2(g2.cpu().numpy(), g1.cpu().numpy()) < 1e-12
    # the mute: a muted trace carries no adjoint source, so masking it changes the gradient
    l3, g3 = whole.misfit_gradient(c, obs, misfit=TraceMisfit(dt_obs, 20.0))
    assert rel_l2(g3.cpu().numpy(), g1.cpu().numpy()) > 1e-6


@pytest.mark.parametrize("n_t,n_tr", [(1, 1), (2, 3), (33, 1), (64, 2), (65, 5)])
def test_short_and_single_traces_against_the_oracle(n_t, n_tr):
    """Edge sizes: one-sample traces, a single trace (no partner in its pair), lengths at the 64-point
    minimum filter and just above it."""
    import misfit_oracle as mo

    rng = np.random.default_rng(n_t * 10 + n_tr)
    obs = rng.standard_normal((n_tr, n_t))
    pred = obs + 0.5 * rng.standard_normal((n_tr, n_t))
    lo, go = mo.band_limited_mse(pred, obs, 0.01, 12.0, 0.3, True, None, sensor=20.0)
    mf = TraceMisfit(0.01, 12.0, 0.3, True, sensor_cutoff=20.0)
    mf.prepare(_t(obs, torch.float64))
    loss, g = mf.value_and_grad(_t(pred, torch.float64))
    assert _rel(loss, lo) < 1e-11
    assert rel_l2(g.cpu().numpy(), go) < 1e-10


@pytest.mark.parametrize("dtype", DTYPES)
def test_filters_are_zero_phase_and_attenuate(dtype):
    """tests/test_photoacoustic3d.py:40-46 and tests/test_instances_wave_family.py:49-55 on the device:
    the pass band comes through without a phase shift, the stop band is removed, a single 1-D trace
    is filtered like a row, and no sensor cutoff returns the input itself."""
    t = torch.arange(200, dtype=torch.float64, device="cuda") * 0.05
    slow, fast = torch.sin(2 * torch.pi * 0.2 * t).to(dtype), torch.sin(2 * torch.pi * 4.0 * t).to(dtype)
    out = gaussian_lowpass(torch.stack([slow, fast]), 0.05, 1.0)
    assert float((out[0] - slow)[20:-20].abs().max()) < 0.05
    assert float(out[1][20:-20].abs().max()) < 1e-3
    single = gaussian_lowpass(slow, 0.05, 1.0)  # no partner trace in its complex pair
    assert single.shape == slow.shape
    assert rel_l2(single.cpu().numpy(), out[0].cpu().numpy()) < TOL[dtype][0]
    assert gaussian_lowpass(slow, 0.05, None) is slow
    dt = 0.004
    t = torch.arange(500, dtype=torch.float64, device="cuda") * dt
    low, high = torch.sin(2 * torch.pi * 2.0 * t), torch.sin(2 * torch.pi * 20.0 * t)
    y = lowpass((low + high).to(dtype), dt, f_max=6.0)
    assert float((y[100:400].double() - low[100:400]).abs().max()) < 0.05
