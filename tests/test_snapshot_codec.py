"""CPU model of the delta16 snapshot codec (nw::d16_encode / nw::d16_decode in
nefi_b200/csrc/aux_kernels.cuh), operation for operation in float32: its int16 codes never
overflow, decoding reproduces the encoder's integer values exactly, and the rounding error is
half a step, on smooth, rough and adversarial blocks."""

from __future__ import annotations

import numpy as np
import pytest

F = np.float32


def encode(x: np.ndarray):
    """x: (n_blocks, 32) float32 -> codes (int64, must fit int16), step, anchor (float32)."""
    x = x.astype(F)
    a = x[:, :1]
    dx = np.zeros_like(x)
    dx[:, 1:] = x[:, 1:] - x[:, :-1]
    d2 = dx.copy()
    d2[:, 2:] = dx[:, 2:] - dx[:, 1:-1]
    m = np.abs(d2).max(1, keepdims=True)
    r = np.abs(x - a).max(1, keepdims=True)
    s = np.maximum(np.maximum(m * F(1.0 / 32000.0), r * F(2.0**-22)), F(1.17549435e-38)).astype(F)
    inv = (F(1) / s).astype(F)
    q = np.rint(((x - a).astype(F) * inv).astype(F)).astype(np.int64)
    qm1 = np.zeros_like(q)
    qm1[:, 1:] = q[:, :-1]
    qm2 = np.zeros_like(q)
    qm2[:, 2:] = q[:, :-2]
    d = q - 2 * qm1 + qm2
    d[:, 0] = 0
    d[:, 1] = q[:, 1]
    return d, s, a, q


def decode(d, s, a):
    q = np.cumsum(np.cumsum(d, 1), 1)
    return (a.astype(np.float64) + s.astype(np.float64) * q.astype(np.float64)).astype(F), q


def blocks(kind: str, rng, n=4096):
    z = np.arange(32)
    if kind == "smooth":
        k = rng.uniform(0.05, 0.6, (n, 1))
        return (rng.uniform(-1, 1, (n, 1)) * np.sin(k * z + rng.uniform(0, 6, (n, 1)))).astype(F)
    if kind == "noise":
        return rng.standard_normal((n, 32)).astype(F)
    if kind == "ramp":  # second differences vanish: the range bound sets the step
        return (rng.uniform(-1e3, 1e3, (n, 1)) + rng.uniform(-50, 50, (n, 1)) * z).astype(F)
    if kind == "spike":
        x = np.zeros((n, 32), F)
        x[np.arange(n), rng.integers(0, 32, n)] = rng.uniform(-1e5, 1e5, n)
        return x
    if kind == "tiny":
        return (rng.standard_normal((n, 32)) * 1e-37).astype(F)
    if kind == "offset":  # a large constant plus a small wave
        return (1e4 + 1e-2 * np.sin(0.3 * z + rng.uniform(0, 6, (n, 1)))).astype(F)
    if kind == "zero":
        return np.zeros((n, 32), F)
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["smooth", "noise", "ramp", "spike", "tiny", "offset", "zero"])
def test_delta16_codes_fit_and_decode_exactly(kind):
    rng = np.random.default_rng(7)
    x = blocks(kind, rng)
    d, s, a, q = encode(x)
    assert np.abs(d).max() <= 32767
    rec, q2 = decode(d, s, a)
    assert np.array_equal(q, q2)                       # two prefix sums undo the second differences
    assert np.abs(q).max() <= 2**22                    # exact in float32 and int32
    err = np.abs(rec.astype(np.float64) - x)
    # half a step from rint, the float32 rounding of (x - a) / s (3 * 2^-24 of |Q| steps), and the one
    # rounding of the decoding fma
    bound = s.astype(np.float64) * (0.5 + 2e-7 * np.abs(q)) + np.abs(x) * 2.0**-23 + 2.0**-149
    assert (err <= bound).all()


def test_delta16_step_follows_the_second_differences_of_smooth_blocks():
    """On smooth blocks the step is set by the second differences, far below a block-maximum scale."""
    rng = np.random.default_rng(8)
    x = blocks("smooth", rng)
    _, s, _, _ = encode(x)
    fixed = np.abs(x).max(1, keepdims=True) / 32767
    ok = np.abs(x).max(1) > 0.05
    assert np.median((s / fixed)[ok]) < 0.5
