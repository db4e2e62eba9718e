"""CPU oracle of the trace misfit: numpy restatement of the reference's band-limited MSE, its low-pass,
the sensors' Gaussian response and the masked mean, with hand-derived gradients.

TEST INFRASTRUCTURE ONLY: used by tests/ and bench.py's CPU baseline as the checker; never by the
``nefi_b200`` product path. Pinned to the reference's own outputs by tests/test_oracle_golden.py.

Follows nefi/instances/wave_fwi/losses.py:28-35 (``_window``), :38-48 (``lowpass``), :78-86
(``BandLimitedMSE.forward``), nefi/instances/photoacoustic3d/sensor.py:24-38 (``gaussian_lowpass``),
nefi/losses/data.py:46-52 (``MSE``), nefi/measurement.py:86-91 (``masked_mean``) and
nefi/utils/tensor.py:21-23 (``next_fast_len``: scipy's real-transform rule, the next 2^a 3^b 5^c).
The gradients use that every filter here is real and even in time (a zero-phase response applied to a
zero-padded trace and cropped), hence its own adjoint.
"""

from __future__ import annotations

import numpy as np


def next_fast_len(n: int) -> int:
    """Smallest 2^a 3^b 5^c >= n (nefi/utils/tensor.py:21-23 with scipy's real=True)."""
    m = max(int(n), 1)
    while True:
        r = m
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def window(n_fft: int, dt: float, f_max: float, taper: float) -> np.ndarray:
    """Cosine roll-off window on the rfft bins (losses.py:28-35)."""
    f = np.fft.rfftfreq(n_fft, d=dt)
    f1 = (1.0 - taper) * f_max
    w = np.ones_like(f)
    roll = (f > f1) & (f < f_max)
    w[roll] = 0.5 * (1.0 + np.cos(np.pi * (f[roll] - f1) / max(f_max - f1, 1e-30)))
    w[f >= f_max] = 0.0
    return w


def _filter(x: np.ndarray, n_fft: int, w: np.ndarray) -> np.ndarray:
    n = x.shape[-1]
    dtype = x.dtype
    y = np.fft.irfft(np.fft.rfft(x.astype(np.float64), n=n_fft, axis=-1) * w, n=n_fft, axis=-1)[..., :n]
    return y.astype(dtype)


def lowpass(x, dt: float, f_max: float, taper: float = 0.3) -> np.ndarray:
    """Zero-phase low-pass along the last axis (losses.py:38-48)."""
    x = np.asarray(x)
    n_fft = next_fast_len(2 * x.shape[-1])
    return _filter(x, n_fft, window(n_fft, dt, f_max, taper))


def gaussian_lowpass(x, dt: float, f_cutoff: float | None) -> np.ndarray:
    """Zero-phase Gaussian ``exp(-(f/f_c)^2 / 2)`` along the last axis (sensor.py:24-38)."""
    x = np.asarray(x)
    if f_cutoff is None or f_cutoff <= 0:
        return x
    size = 2 * x.shape[-1]
    f = np.fft.rfftfreq(size, d=dt)
    return _filter(x, size, np.exp(-0.5 * (f / f_cutoff) ** 2))


def _masked_mean_parts(x2: np.ndarray, mask) -> tuple[float, np.ndarray | float, float]:
    """``masked_mean`` split as (sum, weights, count) (nefi/measurement.py:86-91)."""
    if mask is None:
        return float(x2.sum(dtype=np.float64)), 1.0, float(x2.size)
    m = np.broadcast_to(np.asarray(mask, dtype=np.float64), x2.shape)
    return float((x2 * m).sum()), m, max(float(m.sum()), 1e-12)


def band_limited_mse(pred, obs, dt: float, f_max: float | None, taper: float = 0.3, relative: bool = True,
                     mask=None, sensor: float | None = None) -> tuple[float, np.ndarray]:
    """``BandLimitedMSE`` (losses.py:78-86) of ``G pred`` against ``obs`` (``G`` = the sensor response
    when ``sensor`` is given, else the identity) and its gradient w.r.t. ``pred``; float64 arithmetic."""
    p = np.asarray(pred, dtype=np.float64)
    o = np.asarray(obs, dtype=np.float64)
    r = gaussian_lowpass(p, dt, sensor) - o
    of = o
    if f_max is not None:
        r = lowpass(r, dt, f_max, taper)
        if relative:
            of = lowpass(o, dt, f_max, taper)
    num, m, count = _masked_mean_parts(r * r, mask)
    den = 1.0
    if relative:
        den = max(_masked_mean_parts(of * of, mask)[0] / count, 1e-30)
    loss = num / count / den
    g = (2.0 / (count * den)) * (m * r)
    if f_max is not None:
        g = lowpass(g, dt, f_max, taper)
    return loss, gaussian_lowpass(g, dt, sensor)


def sensor_mse(pred, obs, dt: float, f_cutoff: float, mask=None) -> tuple[np.ndarray, float, np.ndarray]:
    """``MSE`` (nefi/losses/data.py:46-52) of the sensor-filtered prediction: ``(G pred, loss, grad)``."""
    y = gaussian_lowpass(np.asarray(pred, dtype=np.float64), dt, f_cutoff)
    loss, g = band_limited_mse(pred, obs, dt, None, relative=False, mask=mask, sensor=f_cutoff)
    return y, loss, g
