"""Binding to the NEFI operator API when it is importable, with a stand-alone mirror otherwise.

When the ``nefi`` package is on ``sys.path`` the B200 operators subclass
``nefi.operators.base.Operator`` (nefi/operators/base.py:27-78), raise ``nefi.errors`` exception
types (nefi/errors.py:10-27), accept ``nefi.domain.Domain`` objects and register under
``nefi.registry`` (nefi/registry.py:29-47), so ``nefi.invert`` and the instance builders take them
unchanged. Without ``nefi`` (for example on a machine that only has this package) a minimal mirror
with the same names, attributes and exception hierarchy is used, so user code and tests read the
same either way.
"""

from __future__ import annotations

from collections.abc import Mapping, Sequence
from dataclasses import dataclass, field

import torch
from torch import nn

try:  # the reference package is present: bind to it
    from nefi.domain import Domain  # type: ignore
    from nefi.errors import (  # type: ignore
        ConfigError,
        NefiError,
        OperatorError,
        ShapeError,
        SolverError,
    )
    from nefi.losses.data import DataLoss  # type: ignore
    from nefi.operators.base import Operator  # type: ignore
    from nefi.registry import register  # type: ignore

    HAVE_NEFI = True
except Exception:  # pragma: no cover - exercised where nefi is absent
    HAVE_NEFI = False

    class NefiError(Exception):
        """Base class of the errors raised by this package (mirrors ``nefi.errors.NefiError``)."""

    class ShapeError(NefiError, ValueError):
        """Inconsistent tensor or grid shapes."""

    class ConfigError(NefiError, ValueError):
        """Invalid or incomplete configuration."""

    class SolverError(NefiError, RuntimeError):
        """The computation cannot proceed (device-side failure, persistent non-finite values)."""

    class OperatorError(NefiError, RuntimeError):
        """Invalid operator input (for example a wave speed above the CFL bound)."""

    Fields = Mapping[str, torch.Tensor]

    class Operator(nn.Module):
        """Differentiable forward model ``fields -> prediction`` (mirror of the NEFI base class).

        Attributes match ``nefi.operators.base.Operator``: ``primary``, ``homogeneity``,
        ``batchable``, ``traceable``.
        """

        primary: str = "x"
        homogeneity: float | None = None
        batchable: bool = False
        traceable: bool = True

        def forward(self, fields):  # pragma: no cover - abstract
            raise NotImplementedError

        def at_resolution(self, shape: Sequence[int]):
            return self

        def output_shape(self, shape: Sequence[int]):
            return None

        def required_fields(self) -> tuple[str, ...]:
            return (self.primary,)

        def get_field(self, fields, name: str | None = None) -> torch.Tensor:
            name = name or self.primary
            try:
                return fields[name]
            except KeyError as e:
                raise OperatorError(
                    f"{type(self).__name__} needs field {name!r}; available: {tuple(fields)}"
                ) from e

        def apply(self, x: torch.Tensor, **others: torch.Tensor) -> torch.Tensor:
            return self({self.primary: x, **others})

    @dataclass(frozen=True)
    class Domain:
        """Rectangular cell-centred grid: ``shape`` cells over physical ``extent`` per axis."""

        shape: tuple[int, ...]
        extent: tuple[tuple[float, float], ...]
        axes: tuple[str, ...] | None = field(default=None)

        def __post_init__(self) -> None:
            object.__setattr__(self, "shape", tuple(int(s) for s in self.shape))
            ext = tuple((float(lo), float(hi)) for lo, hi in self.extent)
            object.__setattr__(self, "extent", ext)
            if len(ext) != len(self.shape):
                raise ShapeError(f"extent has {len(ext)} axes but shape {self.shape} has "
                                 f"{len(self.shape)}")
            for lo, hi in ext:
                if not hi > lo:
                    raise ShapeError(f"extent must satisfy hi > lo, got {(lo, hi)}")

        @property
        def ndim(self) -> int:
            return len(self.shape)

        def spacing(self, shape=None) -> tuple[float, ...]:
            shape = self.shape if shape is None else tuple(int(s) for s in shape)
            return tuple((hi - lo) / n for (lo, hi), n in zip(self.extent, shape))

        def at(self, shape) -> "Domain":
            shape = (int(shape),) if isinstance(shape, int) else tuple(int(s) for s in shape)
            if len(shape) != self.ndim:
                raise ShapeError(f"shape {shape} does not match domain ndim {self.ndim}")
            return Domain(shape, self.extent, self.axes)

        def physical_coords(self, shape=None, device=None, dtype=None) -> torch.Tensor:
            shape = self.shape if shape is None else tuple(int(s) for s in shape)
            axes = []
            for (lo, hi), n in zip(self.extent, shape):
                i = torch.arange(n, device=device, dtype=dtype or torch.get_default_dtype())
                axes.append(lo + (i + 0.5) * (hi - lo) / n)
            return torch.stack(torch.meshgrid(*axes, indexing="ij"), dim=-1)

    class Loss(nn.Module):
        """A scalar loss term (mirror of ``nefi.losses.base.Loss``, nefi/losses/base.py:53-69)."""

        is_data: bool = False
        step_dependent: bool = False

        def __init__(self, name: str | None = None) -> None:
            super().__init__()
            self.name = name or type(self).__name__.lower()

    class DataLoss(Loss):
        """A data-fidelity term (mirror of ``nefi.losses.data.DataLoss``, nefi/losses/data.py:32-45)."""

        is_data = True

        def __init__(self, name: str | None = None, noise_aware: bool = False) -> None:
            super().__init__(name)
            self.noise_aware = noise_aware

    def register(kind: str, name: str | None = None):
        """No registry without NEFI: the decorator returns the class unchanged."""

        def deco(obj):
            return obj

        return deco


def shape_tuple(shape) -> tuple[int, ...]:
    if isinstance(shape, int):
        return (int(shape),)
    return tuple(int(s) for s in shape)


def resample(x: torch.Tensor, shape: Sequence[int]) -> torch.Tensor:
    """Resample the trailing dims of a known sound-speed map to ``shape``.

    Delegates to ``nefi.utils.tensor.resample`` (nefi/utils/tensor.py:35) when NEFI is present,
    so ``at_resolution`` sees the same map as the reference; otherwise uses area averaging for
    downsampling and (bi/tri)linear interpolation with ``align_corners=False`` for upsampling,
    the convention documented there.
    """
    shape = shape_tuple(shape)
    if HAVE_NEFI:
        from nefi.utils.tensor import resample as _rs  # type: ignore

        return _rs(x, shape)
    d = len(shape)
    old = tuple(x.shape[-d:])
    if old == shape:
        return x
    xb = x.reshape(-1, 1, *old)
    if all(o >= n for o, n in zip(old, shape)):
        pool = {1: torch.nn.functional.adaptive_avg_pool1d, 2: torch.nn.functional.adaptive_avg_pool2d,
                3: torch.nn.functional.adaptive_avg_pool3d}[d]
        y = pool(xb, shape)
    else:
        mode = {1: "linear", 2: "bilinear", 3: "trilinear"}[d]
        y = torch.nn.functional.interpolate(xb, size=shape, mode=mode, align_corners=False)
    return y.reshape(*x.shape[:-d], *shape)


__all__ = [
    "HAVE_NEFI",
    "ConfigError",
    "DataLoss",
    "Domain",
    "NefiError",
    "Operator",
    "OperatorError",
    "ShapeError",
    "SolverError",
    "register",
    "resample",
    "shape_tuple",
]
