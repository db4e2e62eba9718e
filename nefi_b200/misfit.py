"""Fused trace misfit on the device: band-limited (relative) MSE, the sensors' Gaussian response and the
adjoint source they produce, over ``libnefiwave`` (``nw_misfit_prepare`` / ``nw_misfit`` /
``nw_trace_filter``).

Drop-ins:

* :class:`BandLimitedMSEB200` for ``nefi.instances.wave_fwi.losses.BandLimitedMSE``
  (wave_fwi/losses.py:51-86): same constructor and value; its backward is the fused adjoint source.
* :func:`lowpass` / :func:`gaussian_lowpass` for the reference's functions of the same names
  (wave_fwi/losses.py:38-48, photoacoustic3d/sensor.py:24-38).
* :class:`SensorBandwidthB200` for ``nefi.instances.photoacoustic3d.sensor.SensorBandwidth``
  (sensor.py:41-86).
* :class:`TraceMisfit`: loss and ``dLoss/dpred`` in one pass, the adjoint source that
  ``WaveOperatorB200.misfit_gradient(..., misfit=...)`` feeds to the adjoint sweep.

The filters' responses are computed once on the host in float64 from the reference's own windows and
kept on the device; everything per call runs on the current CUDA stream. CPU tensors are an error.
"""

from __future__ import annotations

import ctypes as C
from collections.abc import Sequence

import numpy as np
import torch

from . import _lib
from ._compat import ConfigError, DataLoss, Operator, ShapeError, shape_tuple

__all__ = ["BandLimitedMSEB200", "SensorBandwidthB200", "TraceMisfit", "band_limited_mse", "filter_response",
           "gaussian_lowpass", "lowpass"]

_DT = {torch.float32: 0, torch.float64: 1}
_RESPONSES: dict = {}


def _check(x: torch.Tensor, name: str) -> None:
    if x.device.type != "cuda":
        raise ConfigError(f"{name} must be a CUDA tensor, got {x.device}")
    if x.dtype not in _DT:
        raise ConfigError(f"{name} must be float32 or float64, got {x.dtype}")


def filter_response(kind: int, n_t: int, dt: float, f: float, taper: float, dtype: torch.dtype,
                    device: torch.device) -> torch.Tensor:
    """Device copy of the filter response for ``n_t``-sample traces (cached per arguments)."""
    key = (kind, int(n_t), float(dt), float(f), float(taper), dtype, str(device))
    if key not in _RESPONSES:
        lib = _lib.load()
        k = lib.nw_filter_log2_len(int(n_t))
        host = np.empty(1 << k, dtype=np.float32 if dtype == torch.float32 else np.float64)
        _lib.check(lib.nw_filter_response(kind, int(n_t), float(dt), float(f), float(taper), _DT[dtype],
                                          host.ctypes.data))
        _RESPONSES[key] = torch.from_numpy(host).to(device)
    return _RESPONSES[key]


def _traces(x: torch.Tensor, mask: torch.Tensor | None = None, per_sample: bool = True) -> _lib.Traces:
    n_t = int(x.shape[-1])
    t = _lib.Traces()
    t.dtype = _DT[x.dtype]
    t.n_t = n_t
    t.n_traces = x.numel() // max(n_t, 1)
    t.mask = mask.data_ptr() if mask is not None else None
    t.mask_per_sample = 1 if per_sample else 0
    t.log2_len = _lib.load().nw_filter_log2_len(max(n_t, 1))
    return t


@_lib.on_device
def _apply_filter(x: torch.Tensor, kind: int, dt: float, f: float, taper: float) -> torch.Tensor:
    _check(x, "traces")
    x = x.contiguous()
    y = torch.empty_like(x)
    if x.numel() == 0:
        return y
    resp = filter_response(kind, x.shape[-1], dt, f, taper, x.dtype, x.device)
    _lib.check(_lib.load().nw_trace_filter(C.byref(_traces(x)), x.data_ptr(), resp.data_ptr(), y.data_ptr(),
                                           _lib.stream_handle(x.device)))
    return y


class _Filter(torch.autograd.Function):
    """A zero-phase filter: symmetric, so its backward is the same filter."""

    @staticmethod
    def forward(ctx, x, kind, dt, f, taper):
        ctx.args = (kind, dt, f, taper)
        return _apply_filter(x, kind, dt, f, taper)

    @staticmethod
    def backward(ctx, g):
        return _apply_filter(g, *ctx.args), None, None, None, None


def lowpass(x: torch.Tensor, dt: float, f_max: float, taper: float = 0.3) -> torch.Tensor:
    """Zero-phase low-pass along the last axis: flat to ``(1 - taper) f_max``, cosine roll-off to 0 at
    ``f_max`` (nefi/instances/wave_fwi/losses.py:38-48)."""
    return _Filter.apply(x, _lib.NW_FILTER_LOWPASS, float(dt), float(f_max), float(taper))


def gaussian_lowpass(traces: torch.Tensor, dt: float, f_cutoff: float | None) -> torch.Tensor:
    """Zero-phase Gaussian low-pass ``exp(-(f/f_c)^2 / 2)`` along the last axis; ``f_cutoff`` None or
    <= 0 returns the traces unchanged (nefi/instances/photoacoustic3d/sensor.py:24-38)."""
    if f_cutoff is None or f_cutoff <= 0:
        return traces
    return _Filter.apply(traces, _lib.NW_FILTER_GAUSSIAN, float(dt), float(f_cutoff), 0.0)


class TraceMisfit:
    """``L = masked_mean(|W (G pred - obs)|^2) / masked_mean(|W obs|^2)`` (the denominator only when
    ``relative``) and ``dL/dpred`` in one pass over the traces.

    ``W`` is the low-pass of ``BandLimitedMSE`` (identity when ``f_max`` is None) and ``G`` the sensors'
    Gaussian response of ``SensorBandwidth`` (identity when ``sensor_cutoff`` is None), so ``pred`` is the
    propagator's raw output. :meth:`prepare` fixes the observed data (and mask) once; each
    :meth:`value_and_grad` call then adds one slice of predicted rows. Observations are weighted by
    ``mask`` (broadcastable to ``obs``) as ``Measurement.masked_mean`` does (nefi/measurement.py:86-91).
    """

    def __init__(self, dt: float, f_max: float | None = None, taper: float = 0.3, relative: bool = True,
                 sensor_cutoff: float | None = None) -> None:
        self.dt = float(dt)
        self.f_max = None if f_max is None else float(f_max)
        self.taper = float(taper)
        self.relative = bool(relative)
        self.sensor_cutoff = None if sensor_cutoff is None or sensor_cutoff <= 0 else float(sensor_cutoff)
        self._obs = self._mask = self._state = None
        self._key = None

    def _responses(self, n_t: int, dtype, device):
        w = (filter_response(_lib.NW_FILTER_LOWPASS, n_t, self.dt, self.f_max, self.taper, dtype, device)
             if self.f_max is not None else None)
        g = (filter_response(_lib.NW_FILTER_GAUSSIAN, n_t, self.dt, self.sensor_cutoff, 0.0, dtype, device)
             if self.sensor_cutoff is not None else None)
        return w, g

    @_lib.on_device
    def prepare(self, obs: torch.Tensor, mask: torch.Tensor | None = None, always: bool = False) -> None:
        """Fix the observed traces ``obs`` (``(..., n_t)``, CUDA) and their weights. The observation's
        terms are recomputed only when ``obs`` or ``mask`` changed, or with ``always`` (a caller that
        records the launches in a CUDA graph and refills ``obs`` in place between replays). The state
        array is kept across calls, so its device address does not change."""
        _check(obs, "observed")
        key = (obs.data_ptr(), obs._version, tuple(obs.shape), obs.dtype,
               None if mask is None else (mask.data_ptr(), mask._version, tuple(mask.shape)))
        if key == self._key and not always:
            self._state[_lib.NW_MISFIT_SUM:_lib.NW_MISFIT_LOSS + 1].zero_()
            return
        obs = obs.detach().contiguous()
        m = None
        if mask is not None:
            m = torch.as_tensor(mask).to(device=obs.device, dtype=obs.dtype)
            if m.ndim >= 1 and m.shape[-1] == 1:  # one weight per trace (a trace mute): no per-sample array
                m = m.expand(*obs.shape[:-1], 1)[..., 0].contiguous()
            else:
                m = m.expand_as(obs).contiguous()
        w, _ = self._responses(obs.shape[-1], obs.dtype, obs.device)
        state = self._state
        if state is None or state.device != obs.device:
            state = torch.empty(_lib.NW_MISFIT_STATE, dtype=torch.float64, device=obs.device)
        if obs.numel() == 0:
            raise ShapeError("observed traces are empty")
        _lib.check(_lib.load().nw_misfit_prepare(
            C.byref(_traces(obs, m, m is not None and m.shape == obs.shape)), obs.data_ptr(),
            None if w is None else w.data_ptr(),
            1 if self.relative else 0, state.data_ptr(), _lib.stream_handle(obs.device)))
        self._obs, self._mask, self._state, self._key = obs, m, state, key

    @_lib.on_device
    def value_and_grad(self, pred: torch.Tensor, rows: slice | None = None, want_grad: bool = True,
                       out: torch.Tensor | None = None):
        """Add ``pred`` (the rows ``rows`` of the prepared observation along its first axis, all rows by
        default) to the misfit; returns ``(loss so far, dLoss/dpred)``, the loss a 0-dim float64 view of
        the device state and the gradient in ``pred``'s dtype (None without ``want_grad``), written
        into ``out`` when given (contiguous, ``pred``'s shape and dtype)."""
        if self._state is None:
            raise ConfigError("TraceMisfit.prepare(observed) must come first")
        _check(pred, "pred")
        obs, m = self._obs, self._mask
        if rows is not None:  # the kernels read dense rows: a strided selection is gathered first
            obs = obs[rows].contiguous()
            m = None if m is None else m[rows].contiguous()
        if tuple(pred.shape) != tuple(obs.shape):
            raise ShapeError(f"pred has shape {tuple(pred.shape)}, observed rows {tuple(obs.shape)}")
        if pred.dtype != obs.dtype:
            raise ConfigError(f"pred dtype {pred.dtype} differs from the observed {obs.dtype}")
        if pred.device != obs.device:
            raise ConfigError(f"pred is on {pred.device}, the observed traces on {obs.device}")
        pred = pred.detach().contiguous()
        grad = None
        if want_grad:
            if out is not None:
                if (tuple(out.shape) != tuple(pred.shape) or out.dtype != pred.dtype or not out.is_contiguous()
                        or out.device != pred.device):
                    raise ShapeError("out must be a contiguous tensor of pred's shape, dtype and device")
                grad = out
            else:
                grad = torch.empty_like(pred)
        w, g = self._responses(pred.shape[-1], pred.dtype, pred.device)
        _lib.check(_lib.load().nw_misfit(
            C.byref(_traces(pred, m, m is not None and m.shape == pred.shape)), pred.data_ptr(), obs.data_ptr(), None if g is None else g.data_ptr(),
            None if w is None else w.data_ptr(), self._state.data_ptr(), None if grad is None else grad.data_ptr(),
            _lib.stream_handle(pred.device)))
        return self._state[_lib.NW_MISFIT_LOSS], grad


class _MisfitFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pred, misfit: TraceMisfit):
        misfit._state[_lib.NW_MISFIT_SUM:_lib.NW_MISFIT_LOSS + 1].zero_()
        loss, grad = misfit.value_and_grad(pred, want_grad=pred.requires_grad)
        if grad is not None:
            ctx.save_for_backward(grad)
        return loss.to(pred.dtype, copy=True)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return grad * g.to(grad.dtype), None


def band_limited_mse(pred: torch.Tensor, obs: torch.Tensor, dt: float, f_max: float | None,
                     taper: float = 0.3, relative: bool = True, mask: torch.Tensor | None = None) -> torch.Tensor:
    """``BandLimitedMSE``'s value as a differentiable function of ``pred`` (losses.py:78-86)."""
    mf = TraceMisfit(dt, f_max, taper, relative)
    mf.prepare(obs, mask)
    return _MisfitFunction.apply(pred, mf)


class BandLimitedMSEB200(DataLoss):
    """Drop-in for ``BandLimitedMSE`` (nefi/instances/wave_fwi/losses.py:51-86):
    ``L = mean(|lowpass(pred - obs)|^2) / mean(|lowpass(obs)|^2)`` over observed entries, the
    denominator only with ``relative``, no filter when ``f_max`` is None. The observation's terms are
    computed once per observed tensor; the value and its gradient take one fused pass per call."""

    def __init__(self, f_max: float | None, dt: float, taper: float = 0.3, relative: bool = True,
                 name: str | None = None) -> None:
        super().__init__(name)
        self.f_max = None if f_max is None else float(f_max)
        self.dt = float(dt)
        self.taper = float(taper)
        self.relative = relative
        self._misfit = TraceMisfit(self.dt, self.f_max, self.taper, relative)

    def forward(self, ctx) -> torch.Tensor:
        self._misfit.prepare(ctx.obs.data, getattr(ctx.obs, "mask", None))
        return _MisfitFunction.apply(ctx.pred, self._misfit)

    def extra_repr(self) -> str:
        return f"f_max={self.f_max}, dt={self.dt}, relative={self.relative}"


class SensorBandwidthB200(Operator):
    """Drop-in for ``SensorBandwidth`` (nefi/instances/photoacoustic3d/sensor.py:41-86): wraps a trace
    operator with the sensors' zero-phase Gaussian response, applied (and differentiated) on the
    device."""

    traceable = False

    def __init__(self, inner: Operator, dt_obs: float, f_cutoff: float | None) -> None:
        super().__init__()
        self.inner = inner
        self.primary = inner.primary
        self.homogeneity = inner.homogeneity
        self.dt_obs = float(dt_obs)
        self.f_cutoff = None if f_cutoff is None or f_cutoff <= 0 else float(f_cutoff)
        tag = getattr(inner, "fidelity_tag", type(inner).__name__)
        self.fidelity_tag = f"{tag}-lp{self.f_cutoff:g}" if self.f_cutoff else str(tag)
        self._res: dict = {}

    def forward(self, fields) -> torch.Tensor:
        return gaussian_lowpass(self.inner(fields), self.dt_obs, self.f_cutoff)

    def at_resolution(self, shape: Sequence[int]) -> "SensorBandwidthB200":
        shape = shape_tuple(shape)
        inner = self.inner.at_resolution(shape)
        if inner is self.inner:
            return self
        if shape not in self._res:
            op = SensorBandwidthB200(inner, self.dt_obs, self.f_cutoff)
            op.fidelity_tag = self.fidelity_tag
            self._res[shape] = op
        return self._res[shape]

    def output_shape(self, shape: Sequence[int]):
        return self.inner.output_shape(shape)

    def required_fields(self) -> tuple[str, ...]:
        return self.inner.required_fields()

    def extra_repr(self) -> str:
        return f"f_cutoff={self.f_cutoff}, dt_obs={self.dt_obs:g}"
