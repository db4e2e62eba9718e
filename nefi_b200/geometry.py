"""Host-side geometry of the padded leapfrog grid, computed in float64 on the CPU.

Everything here is derived once per operator (and per resolution) and handed to the CUDA library
as small tables: padded extents, the Laplacian weights, the absorbing-layer coefficients, the
multilinear source/receiver stencils and the CFL time axis. The formulas follow the reference's
conventions so that the device path sees bit-identical constants:

* padded extent ``P = n + 2a`` with ``a = ceil(W/h - 1e-9)`` per axis, cell centres at
  ``lo_pad + (i + 1/2) h`` (nefi/physics/wave.py:204-216, nefi/domain.py:108-118);
* relative layer depth ``xi`` at cell centres (nefi/physics/wave.py:248-261);
* sponge ``A = 1/(1 + sigma dt/2)``, ``B = 1 - sigma dt/2`` with
  ``sigma = sum_ax 3 c_max ln(1/R)/(a_ax h_ax) xi_ax^2`` (nefi/physics/wave.py:431-447, 469-472);
* Cerjan taper ``exp(-(gamma max_ax xi_ax)^2)`` (nefi/physics/wave.py:473-475);
* Laplacian weights ``[1,-2,1]/h^2`` or ``[-1/12,4/3,-5/2,4/3,-1/12]/h^2`` per axis summed into
  one stencil (nefi/physics/wave.py:121-141);
* CFL step ``courant * 2 / (c_max sqrt(sum rho/h^2))`` with ``rho = 4`` (order 2) or ``16/3``
  (order 4), ``substeps = ceil(dt_obs/dt_max - 1e-12)`` (nefi/physics/timestep.py:177-207,
  nefi/physics/wave.py:394-397);
* multilinear point stencils with ``u = (x - lo_pad)/h - 1/2`` and the lower corner clamped to
  ``P - 2`` (nefi/physics/wave.py:272-300); source weights ``w / cell_volume * dt^2``
  (nefi/physics/wave.py:312-318, 670-674);
* Ricker wavelet ``(1 - 2 a^2) exp(-a^2)``, ``a = pi f0 (t - t0)`` (nefi/physics/wave.py:101-111).
"""

from __future__ import annotations

import math
from collections.abc import Sequence

import torch

from ._compat import ConfigError, ShapeError

ABSORBING = ("pml", "sponge", "cerjan", "none")
GRAD_MODES = ("checkpoint", "autograd")

# One-sided second-derivative coefficients per accuracy order: (centre, +-1, +-2).
STENCIL = {2: (-2.0, 1.0), 4: (-5.0 / 2.0, 4.0 / 3.0, -1.0 / 12.0)}
# max |symbol| * h^2 of the 1-D stencils (von Neumann), per order.
LAPLACIAN_RHO = {2: 4.0, 4: 16.0 / 3.0}


def ricker(t: torch.Tensor, f0: float, t0: float | None = None) -> torch.Tensor:
    """Ricker wavelet ``(1 - 2a^2) exp(-a^2)`` with ``a = pi f0 (t - t0)``, ``t0 = 1.2/f0``."""
    t0 = 1.2 / f0 if t0 is None else t0
    a2 = (math.pi * f0 * (t - t0)) ** 2
    return (1.0 - 2.0 * a2) * torch.exp(-a2)


def laplacian_eig_max(spacing: Sequence[float], order: int) -> float:
    if order not in LAPLACIAN_RHO:
        raise ConfigError(f"Laplacian order must be 2 or 4, got {order}")
    return sum(LAPLACIAN_RHO[order] / float(h) ** 2 for h in spacing)


def stable_dt(c_max: float, spacing: Sequence[float], order: int = 4, courant: float = 0.9) -> float:
    """Largest stable leapfrog step times the safety factor ``courant``."""
    if not 0.0 < courant <= 1.0:
        raise ConfigError(f"courant safety factor must be in (0, 1], got {courant}")
    if c_max <= 0:
        raise ConfigError(f"c_max must be positive, got {c_max}")
    return float(courant) * 2.0 / (float(c_max) * math.sqrt(laplacian_eig_max(spacing, order)))


def stencil_weights(spacing: Sequence[float], order: int) -> tuple[float, list[float], list[float]]:
    """``(centre, w1[ax], w2[ax])`` of the summed per-axis Laplacian stencil, in float64.

    The centre weight is accumulated axis by axis starting from 0.0, the order in which the
    reference builds its convolution kernel, so the float32 cast matches it exactly.
    """
    if order not in STENCIL:
        raise ConfigError(f"Laplacian order must be 2 or 4, got {order}")
    co = STENCIL[order]
    centre = 0.0
    w1, w2 = [], []
    for h in spacing:
        h2 = float(h) ** 2
        centre += co[0] / h2
        w1.append(co[1] / h2)
        w2.append(co[2] / h2 if order == 4 else 0.0)
    return centre, w1, w2


class PaddedGrid:
    """The simulation grid: the field grid plus an absorbing layer of ``n_abs[ax]`` cells.

    Args:
        domain: the field's domain (``shape``, ``extent``, ``spacing()``).
        absorb_width: physical width of the absorbing layer (0 gives no padding).
    """

    def __init__(self, domain, absorb_width: float = 0.0) -> None:
        self.domain = domain
        self.spacing = tuple(float(h) for h in domain.spacing())
        self.d = len(domain.shape)
        self.n_abs = tuple(
            int(math.ceil(float(absorb_width) / h - 1e-9)) if absorb_width > 0 else 0
            for h in self.spacing
        )
        self.shape = tuple(int(n) for n in domain.shape)
        self.padded_shape = tuple(n + 2 * a for n, a in zip(self.shape, self.n_abs))
        self.lo_pad = tuple(lo - a * h for (lo, _), a, h in zip(domain.extent, self.n_abs, self.spacing))

    @property
    def cell_volume(self) -> float:
        return math.prod(self.spacing)

    @property
    def cells(self) -> int:
        return math.prod(self.padded_shape)

    def layer_depth(self, ax: int, faces: bool = False) -> torch.Tensor:
        """Relative depth ``xi`` in ``[0, 1]`` into the layer along ``ax`` (float64)."""
        a, n = self.n_abs[ax], self.shape[ax]
        m = n + 2 * a + (1 if faces else 0)
        pos = torch.arange(m, dtype=torch.float64)
        if not faces:
            pos = pos + 0.5
        if a == 0:
            return torch.zeros(m, dtype=torch.float64)
        return torch.clamp(torch.maximum(a - pos, pos - (a + n)), min=0.0) / a

    def _broadcast(self, v: torch.Tensor, ax: int) -> torch.Tensor:
        view = [1] * self.d
        view[ax] = -1
        return v.view(view)

    def crop(self, x: torch.Tensor) -> torch.Tensor:
        idx = [slice(None)] * (x.ndim - self.d)
        idx += [slice(a, a + n) for a, n in zip(self.n_abs, self.shape)]
        return x[tuple(idx)]

    def pad(self, x: torch.Tensor, mode: str = "replicate") -> torch.Tensor:
        """Host-side padding (replicate for material maps, zeros otherwise); used for checks.

        Padded cell ``i`` of an axis with layer width ``a`` and ``n`` physical cells holds physical
        cell ``i - a`` (zeros), or the nearest physical cell ``clamp(i - a, 0, n - 1)`` (replicate)."""
        if not any(self.n_abs):
            return x
        for ax, a in enumerate(self.n_abs):
            if a == 0:
                continue
            dim = x.ndim - self.d + ax
            n = x.shape[dim]
            src = torch.arange(-a, n + a, device=x.device)
            if mode == "zeros":
                shape = list(x.shape)
                shape[dim] = n + 2 * a
                out = x.new_zeros(shape)
                out.narrow(dim, a, n).copy_(x)
                x = out
            else:
                x = x.index_select(dim, src.clamp(0, n - 1))
        return x

    def point_stencils(self, points: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """Multilinear stencils of physical ``points (n, d)``: ``(corner (n, d) int64, w (n, 2^d))``.

        ``corner`` is the lower cell index per axis; weight ``k`` belongs to the corner offset
        whose bits (axis 0 most significant) are the binary digits of ``k``, the ordering of the
        reference's flattened stencils. Raises ``ConfigError`` for points outside the grid.
        """
        pts = torch.as_tensor(points, dtype=torch.float64)
        if pts.ndim != 2 or pts.shape[1] != self.d:
            raise ShapeError(f"points must have shape (n, {self.d}), got {tuple(pts.shape)}")
        corners, w_axes = [], []
        for ax in range(self.d):
            h, lo, m = self.spacing[ax], self.lo_pad[ax], self.padded_shape[ax]
            u = (pts[:, ax] - lo) / h - 0.5
            if bool((u < -1e-9).any()) or bool((u > m - 1 + 1e-9).any()):
                raise ConfigError(
                    f"point outside the simulation grid along axis {ax}: coordinates "
                    f"{pts[:, ax].tolist()} vs grid [{lo + 0.5 * h}, {lo + (m - 0.5) * h}]"
                )
            u = u.clamp(0.0, m - 1)
            i0 = torch.floor(u).clamp(max=max(m - 2, 0)).long()
            t = u - i0
            corners.append(i0)
            w_axes.append(torch.stack([1.0 - t, t], dim=1))
        weight = torch.ones(pts.shape[0], 1, dtype=torch.float64)
        for ax in range(self.d):
            weight = (weight[:, :, None] * w_axes[ax][:, None, :]).flatten(1)
        return torch.stack(corners, dim=1), weight

    def flat_indices(self, corner: torch.Tensor) -> torch.Tensor:
        """Row-major flat indices ``(n, 2^d)`` of a stencil's corners on the padded grid."""
        strides = [math.prod(self.padded_shape[ax + 1:]) for ax in range(self.d)]
        out = torch.zeros(corner.shape[0], 1, dtype=torch.long)
        for ax in range(self.d):
            hi = (corner[:, ax] + 1).clamp(max=self.padded_shape[ax] - 1)
            pair = torch.stack([corner[:, ax], hi], 1)
            out = (out[:, :, None] + strides[ax] * pair[:, None, :]).flatten(1)
        return out

    def nearest_index(self, points: torch.Tensor) -> torch.Tensor:
        """Flat padded-grid index of the cell containing each point: per axis the cell whose
        faces ``lo + [i, i + 1) h`` enclose the coordinate, clamped to the padded grid, combined
        with the row-major strides of the padded shape."""
        pts = torch.as_tensor(points, dtype=torch.float64)
        lo = torch.tensor(self.lo_pad[: self.d], dtype=torch.float64)
        h = torch.tensor(self.spacing[: self.d], dtype=torch.float64)
        hi = torch.tensor(self.padded_shape[: self.d], dtype=torch.long) - 1
        cell = torch.minimum(torch.floor((pts - lo) / h).long().clamp(min=0), hi)
        strides = [1] * self.d
        for ax in range(self.d - 2, -1, -1):
            strides[ax] = strides[ax + 1] * self.padded_shape[ax + 1]
        return (cell * torch.tensor(strides, dtype=torch.long)).sum(1)


def as_points(x, d: int, name: str) -> torch.Tensor:
    t = torch.as_tensor(x, dtype=torch.float64)
    if t.ndim == 1 and d == 1:
        t = t[:, None]
    if t.ndim != 2 or t.shape[1] != d:
        raise ShapeError(f"{name} must have shape (n, {d}), got {tuple(t.shape)}")
    return t


class TimeAxis:
    """Observation times ``j * dt_obs`` (``j < n_t``) on a CFL-limited simulation step."""

    def __init__(self, n_t: int, dt_obs: float, c_max: float, spacing, order: int, courant: float):
        self.n_t, self.dt_obs = int(n_t), float(dt_obs)
        dt_max = stable_dt(c_max, spacing, order, courant)
        self.substeps = max(1, int(math.ceil(self.dt_obs / dt_max - 1e-12)))
        self.dt = self.dt_obs / self.substeps
        self.n_steps = (self.n_t - 1) * self.substeps


def damping_rate(grid: PaddedGrid, c_max: float, absorb_R: float) -> torch.Tensor:
    """Sponge damping rate ``sigma`` (1/s) on the padded grid (float64)."""
    sig = torch.zeros(grid.padded_shape, dtype=torch.float64)
    for ax, a in enumerate(grid.n_abs):
        if a:
            smax = 3.0 * c_max * math.log(1.0 / absorb_R) / (a * grid.spacing[ax])
            sig = sig + smax * grid._broadcast(grid.layer_depth(ax), ax) ** 2
    return sig


def sponge_coefficients(grid: PaddedGrid, c_max: float, absorb_R: float, dt: float):
    """float64 ``(A, B)`` of the sponge layer on the padded grid (``None`` without a layer)."""
    if not any(grid.n_abs):
        return None
    half = 0.5 * damping_rate(grid, c_max, absorb_R) * dt
    return 1.0 / (1.0 + half), 1.0 - half


def cerjan_taper(grid: PaddedGrid, gamma: float):
    """float64 Cerjan taper on the padded grid (``None`` without a layer)."""
    if not any(grid.n_abs):
        return None
    xi = torch.stack([grid._broadcast(grid.layer_depth(ax), ax).expand(grid.padded_shape)
                      for ax in range(grid.d)]).amax(0)
    return torch.exp(-((gamma * xi) ** 2))


def pml_profile(grid: PaddedGrid, ax: int, c_max: float, absorb_R: float, faces: bool = False):
    """PML stretching rate ``zeta = 1.5 c_max ln(1/R)/(a h) xi^2`` along ``ax`` (float64, 1-D)."""
    if grid.n_abs[ax] == 0:
        return grid.layer_depth(ax, faces) * 0.0
    zmax = 1.5 * c_max * math.log(1.0 / absorb_R) / (grid.n_abs[ax] * grid.spacing[ax])
    return zmax * grid.layer_depth(ax, faces) ** 2


def pml_coefficients(grid: PaddedGrid, c_max: float, absorb_R: float, dt: float) -> dict:
    """float64 coefficients of the 2-D PML step (nefi/physics/wave.py:476-501): on cells
    ``A = 1/(1 + dt/2 sum zeta)``, ``B = 1 - dt/2 sum zeta``, ``ZZ = dt^2 zeta_x zeta_z``; per axis on
    its ``P+1`` faces ``alpha = (1 - dt/2 zeta_f)/(1 + dt/2 zeta_f)`` and
    ``beta = dt (zeta_other - zeta_f) / ((1 + dt/2 zeta_f) h)`` (``zeta_other`` at the cell
    centres of the other axis)."""
    zc = [grid._broadcast(pml_profile(grid, ax, c_max, absorb_R), ax) for ax in range(2)]
    zsum = (zc[0] + zc[1]).expand(grid.padded_shape)
    out = {"A": 1.0 / (1.0 + 0.5 * dt * zsum), "B": 1.0 - 0.5 * dt * zsum,
           "ZZ": (dt**2 * zc[0] * zc[1]).expand(grid.padded_shape), "alpha": [], "beta": []}
    for ax in range(2):
        zf = grid._broadcast(pml_profile(grid, ax, c_max, absorb_R, faces=True), ax)
        fshape = list(grid.padded_shape)
        fshape[ax] += 1
        den = 1.0 + 0.5 * dt * zf
        out["alpha"].append(((1.0 - 0.5 * dt * zf) / den).expand(fshape))
        out["beta"].append((dt * (zc[1 - ax] - zf) / (den * grid.spacing[ax])).expand(fshape))
    return out
