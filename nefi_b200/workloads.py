"""Seeded synthetic FWI / photoacoustic workloads with the shapes of the benchmark configurations.

No public dataset exists for this path; every model here is generated from a seed with the sizes and
value ranges of the named configuration:

* ``fwi_plain_128``: 128^2 grid, h = 10 m, 2000 m/s + two +-300 m/s Gaussian anomalies (sigma 8
  cells), 20-cell sponge, one 15 Hz Ricker at top centre, 128 receivers on row 2, Courant 0.4,
  1000 steps.
* ``fwi_512``: 512^2, h = 10 m, 6-10 flat/dipping layers 1500-4500 m/s + 4 Gaussian anomalies,
  16 Ricker shots at 10 Hz evenly along the surface, 512 receivers, 4000 steps.
* ``fwi_2048``: 2048^2, layered + salt body (random polygon, 4500 m/s), 32 shots at 12 Hz, 2048
  receivers, 8000 steps.
* ``pat_256``: 256^3, 1500 m/s +-5 % smooth perturbation, 20 random ellipsoids of amplitude
  U[0.2, 1], a 256 x 256 sensor plane on one face, 2000 steps.

Depth is the last (contiguous) axis, as in NEFI's ``wave_fwi`` (axes ``("x", "z")``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from ._compat import Domain


@dataclass
class FWIWorkload:
    name: str
    n: int
    h: float
    c: np.ndarray               # (n, n) m/s
    sources: np.ndarray         # (n_src, 2)
    receivers: np.ndarray       # (n_rec, 2)
    f0: float
    n_steps: int
    courant_number: float = 0.4
    absorb_cells: int = 20
    order: int = 4
    extra: dict = field(default_factory=dict)

    @property
    def domain(self) -> Domain:
        L = self.n * self.h
        return Domain((self.n, self.n), ((0.0, L), (0.0, L)), axes=("x", "z"))

    @property
    def c_max(self) -> float:
        return float(self.c.max())

    @property
    def dt(self) -> float:
        return self.courant_number * self.h / self.c_max

    def operator_kwargs(self) -> dict:
        """Arguments of ``WaveOperator`` reproducing the configuration with one substep per sample."""
        return dict(n_t=self.n_steps + 1, dt_obs=self.dt, f0=self.f0, c_max=self.c_max, order=self.order,
                    absorbing="sponge", absorb_width=self.absorb_cells * self.h, courant=1.0)

    def padded_cells(self) -> int:
        return (self.n + 2 * self.absorb_cells) ** 2


def _surface(n, h, n_src, n_rec):
    L = n * h
    src = np.stack([(np.arange(n_src) + 0.5) * L / n_src, np.full(n_src, 1.5 * h)], 1)
    rec = np.stack([(np.arange(n_rec) + 0.5) * L / n_rec, np.full(n_rec, 2.5 * h)], 1)
    return src, rec


def layered_model(n: int, h: float, rng: np.random.Generator, n_layers=(6, 10), vmin=1500.0,
                  vmax=4500.0, n_anomalies=4) -> np.ndarray:
    """Flat/dipping layers with tanh-smoothed interfaces plus Gaussian anomalies (m/s)."""
    L = n * h
    x = (np.arange(n) + 0.5) * h
    X, Z = np.meshgrid(x, x, indexing="ij")
    k = int(rng.integers(n_layers[0], n_layers[1] + 1))
    depths = np.sort(rng.uniform(0.08, 0.95, k - 1)) * L
    dips = np.tan(np.deg2rad(rng.uniform(-8.0, 8.0, k - 1)))
    vel = np.sort(rng.uniform(vmin, vmax, k))
    c = np.full((n, n), vel[0])
    for d0, dip, v1, v0 in zip(depths, dips, vel[1:], vel[:-1]):
        iface = d0 + dip * (X - 0.5 * L)
        c = c + (v1 - v0) * 0.5 * (1.0 + np.tanh((Z - iface) / (1.5 * h)))
    for _ in range(n_anomalies):
        cx, cz = rng.uniform(0.2, 0.8, 2) * L
        amp = rng.choice([-1.0, 1.0]) * rng.uniform(100.0, 300.0)
        sig = rng.uniform(4.0, 12.0) * h
        c = c + amp * np.exp(-((X - cx) ** 2 + (Z - cz) ** 2) / (2 * sig**2))
    return np.clip(c, vmin, vmax)


def salt_body(c: np.ndarray, h: float, rng: np.random.Generator, v_salt=4500.0) -> np.ndarray:
    """Overwrite a random star-shaped polygon (the salt body) with ``v_salt``."""
    n = c.shape[0]
    L = n * h
    x = (np.arange(n) + 0.5) * h
    X, Z = np.meshgrid(x, x, indexing="ij")
    cx, cz = rng.uniform(0.35, 0.65) * L, rng.uniform(0.4, 0.6) * L
    m = int(rng.integers(7, 13))
    ang = np.sort(rng.uniform(0, 2 * np.pi, m))
    rad = rng.uniform(0.08, 0.22, m) * L
    th = np.arctan2(Z - cz, X - cx) % (2 * np.pi)
    r = np.hypot(X - cx, Z - cz)
    # piecewise-linear boundary radius between the polygon vertices
    ang_ext = np.concatenate([ang - 2 * np.pi, ang, ang + 2 * np.pi])
    rad_ext = np.concatenate([rad, rad, rad])
    rb = np.interp(th, ang_ext, rad_ext)
    out = c.copy()
    out[r < rb] = v_salt
    return out


def fwi_plain_128(seed: int = 0) -> FWIWorkload:
    n, h = 128, 10.0
    g = torch.Generator().manual_seed(seed)
    xs = (torch.arange(n, dtype=torch.float64) + 0.5) * h
    X, Z = torch.meshgrid(xs, xs, indexing="ij")
    c = torch.full((n, n), 2000.0, dtype=torch.float64)
    for s in (1.0, -1.0):
        ctr = torch.rand(2, generator=g, dtype=torch.float64) * n * h * 0.5 + n * h * 0.25
        c = c + s * 300.0 * torch.exp(-((X - ctr[0]) ** 2 + (Z - ctr[1]) ** 2) / (2 * (8 * h) ** 2))
    src = np.array([[n * h / 2, 1.5 * h]])
    rec = np.array([[(i + 0.5) * h, 2.5 * h] for i in range(n)])
    return FWIWorkload("fwi_plain_128", n, h, c.numpy(), src, rec, 15.0, 1000)


def fwi_512(seed: int = 0, n_shots: int = 16, n_steps: int = 4000) -> FWIWorkload:
    n, h = 512, 10.0
    rng = np.random.default_rng(seed)
    c = layered_model(n, h, rng)
    src, rec = _surface(n, h, n_shots, 512)
    return FWIWorkload("fwi_512", n, h, c, src, rec, 10.0, n_steps)


def fwi_2048(seed: int = 0, n_shots: int = 32, n_steps: int = 8000) -> FWIWorkload:
    n, h = 2048, 10.0
    rng = np.random.default_rng(seed)
    c = salt_body(layered_model(n, h, rng), h, rng)
    src, rec = _surface(n, h, n_shots, 2048)
    return FWIWorkload("fwi_2048", n, h, c, src, rec, 12.0, n_steps)


def fwi_salt(n: int = 192, n_shots: int = 32, n_steps: int = 1000, seed: int = 3) -> FWIWorkload:
    """``fwi_2048``'s model family (layers + salt body, 12 Hz, receivers every other cell) on a
    smaller grid: the size at which a float64 CPU run checks the checkpointed 16-bit gradient."""
    h = 10.0
    rng = np.random.default_rng(seed)
    c = salt_body(layered_model(n, h, rng), h, rng)
    src, rec = _surface(n, h, n_shots, n // 2)
    return FWIWorkload(f"fwi_salt_{n}", n, h, c, src, rec, 12.0, n_steps)


def fwi_batch_problems(seed: int = 0, n_problems: int = 64):
    """The uneven batch: grid sizes from {256, 384, 512, 768}^2, 4-16 shots, 1500-6000 steps."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_problems):
        n = int(rng.choice([256, 384, 512, 768]))
        shots = int(rng.integers(4, 17))
        steps = int(rng.integers(1500, 6001))
        c = layered_model(n, 10.0, rng)
        src, rec = _surface(n, 10.0, shots, n)
        out.append(FWIWorkload(f"problem{k}", n, 10.0, c, src, rec, 10.0, steps))
    return out


@dataclass
class PATWorkload:
    name: str
    n: int
    h: float
    c: np.ndarray      # (n, n, n)
    p0: np.ndarray     # (batch, n, n, n)
    sensors: np.ndarray
    n_steps: int
    absorb_cells: int = 20
    order: int = 2
    courant_number: float = 0.3

    @property
    def domain(self) -> Domain:
        L = self.n * self.h
        return Domain((self.n,) * 3, ((0.0, L),) * 3, axes=("x", "y", "z"))

    @property
    def dt(self) -> float:
        return self.courant_number * self.h / float(self.c.max())

    def operator_kwargs(self) -> dict:
        return dict(n_t=self.n_steps + 1, dt_obs=self.dt, c=torch.tensor(self.c), order=self.order,
                    absorbing="sponge", absorb_width=self.absorb_cells * self.h, courant=1.0)


def pat_volume(n: int = 256, batch: int = 4, n_steps: int = 2000, seed: int = 0, h: float = 1e-4,
               n_sensors: int | None = None) -> PATWorkload:
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    pert = np.zeros((n, n, n))
    for _ in range(6):
        k = rng.uniform(1.0, 3.0, 3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        pert += np.sin(2 * np.pi * k[0] * X + ph[0]) * np.sin(2 * np.pi * k[1] * Y + ph[1]) * np.sin(
            2 * np.pi * k[2] * Z + ph[2])
    pert /= np.abs(pert).max()
    c = 1500.0 * (1.0 + 0.05 * pert)
    p0 = np.zeros((batch, n, n, n), dtype=np.float32)
    for b in range(batch):
        for _ in range(20):
            ctr = rng.uniform(0.15, 0.85, 3)
            ax = rng.uniform(0.02, 0.08, 3)
            amp = rng.uniform(0.2, 1.0)
            inside = ((X - ctr[0]) / ax[0]) ** 2 + ((Y - ctr[1]) / ax[1]) ** 2 + ((Z - ctr[2]) / ax[2]) ** 2 <= 1
            p0[b][inside] = np.maximum(p0[b][inside], amp)
    m = n if n_sensors is None else n_sensors
    L = n * h
    s = (np.arange(m) + 0.5) * L / m
    SX, SY = np.meshgrid(s, s, indexing="ij")
    sensors = np.stack([SX.ravel(), SY.ravel(), np.full(m * m, 0.5 * h)], -1)
    return PATWorkload("pat_256" if n == 256 else f"pat_{n}", n, h, c, p0, sensors, n_steps)


WORKLOADS = {"fwi_plain_128": fwi_plain_128, "fwi_512": fwi_512, "fwi_2048": fwi_2048}


def cell_updates(w: FWIWorkload, n_shots: int | None = None) -> int:
    """Useful cell-updates of one shot-gradient sweep: forward + adjoint over the padded grid."""
    s = len(w.sources) if n_shots is None else n_shots
    return 2 * w.padded_cells() * w.n_steps * s


__all__ = ["FWIWorkload", "PATWorkload", "WORKLOADS", "cell_updates", "fwi_2048", "fwi_512",
           "fwi_batch_problems", "fwi_salt", "fwi_plain_128", "layered_model", "pat_volume", "salt_body"]
