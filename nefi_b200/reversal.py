"""Classical photoacoustic baseline: time reversal of receiver traces (``time_reversal``).

Same signature, modes and errors as ``nefi.physics.wave.time_reversal`` (nefi/physics/wave.py:878-968):

* ``mode="dirichlet"`` (k-Wave style): from rest, the receivers' nearest cells are held at the traces
  at reversed time ``T - n dt`` (linear in time between samples) after every step; the cropped field
  at ``t = 0`` estimates ``p0``. The whole loop runs on the GPU (``nw_time_reversal``).
* ``mode="adjoint"``: the exact discrete adjoint of ``WaveInitialConditionOperatorB200`` applied to
  the traces (reverse mode through the operator).
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._compat import ConfigError, ShapeError
from .operators import WaveInitialConditionOperatorB200, _Run
from .plan import ghost_view


@torch.no_grad()
@_lib.on_device
def time_reversal(traces, domain, receivers, *, dt_obs: float, c=1.0, mode: str = "dirichlet", order: int = 4,
                  absorbing: str = "pml", absorb_width: float | None = None, absorb_R: float = 1e-3,
                  courant: float = 0.9) -> torch.Tensor:
    """Time-reversal reconstruction of an initial pressure from ``traces`` ``(n_receivers, n_t)``
    sampled at ``t_j = j dt_obs`` (a leading batch dimension of one is accepted); returns the
    ``p0`` estimate on ``domain.shape`` in the traces' dtype, on their (CUDA) device."""
    if mode not in ("dirichlet", "adjoint"):
        raise ConfigError(f"mode must be 'dirichlet' or 'adjoint', got {mode!r}")
    tr = torch.as_tensor(traces)
    if tr.ndim == 3 and tr.shape[0] == 1:
        tr = tr[0]
    if tr.ndim != 2:
        raise ShapeError(f"traces must be (n_receivers, n_t), got {tuple(tr.shape)}")
    device = tr.device
    dtype = tr.dtype if tr.is_floating_point() else torch.float32
    tr = tr.to(dtype)
    op = WaveInitialConditionOperatorB200(domain, receivers, n_t=tr.shape[-1], dt_obs=dt_obs, c=c, order=order,
                                          absorbing=absorbing, absorb_width=absorb_width, absorb_R=absorb_R,
                                          courant=courant, grad_mode="autograd")
    if mode == "adjoint":
        with torch.enable_grad():
            p0 = torch.zeros(tuple(domain.shape), device=device, dtype=dtype, requires_grad=True)
            (grad,) = torch.autograd.grad((op({"p0": p0}) * tr).sum(), p0)
        return grad
    op._check_device(tr, "traces")
    if tr.shape[0] != op.receivers.shape[0]:
        raise ShapeError(f"traces have {tr.shape[0]} rows for {op.receivers.shape[0]} receivers")
    plan = op._plan(device, dtype)
    _, c2dt2 = op._known_speed(device, dtype)
    medium = plan.medium(c2dt2)
    acq = plan.acquisition(1)
    run = _Run(plan, 1, op.n_steps, ("ring", None), "exact")
    # the receivers' cells (nefi/physics/wave.py:302-310); where several share a cell the last one's
    # trace holds it, as the reference's sequential index assignment leaves it
    flat = op.grid.nearest_index(op.receivers)
    last = {}
    for r, f in enumerate(flat.tolist()):
        last[f] = r
    rows = torch.tensor(sorted(last.values()), dtype=torch.long)
    P = op.grid.padded_shape
    idx = flat[rows]
    off = torch.full_like(idx, int(plan.g.origin))
    for ax in reversed(range(len(P))):
        off += (idx % P[ax]) * int(plan.g.stride[ax])
        idx = idx // P[ax]
    cells = off.to(device)
    tr_sel = tr[rows.to(device)].contiguous()
    s = _lib.stream_handle(device)
    _lib.check(_lib.load().nw_time_reversal(C.byref(plan.g), C.byref(medium), C.byref(acq), C.byref(plan.time),
                                            C.byref(run.storage), C.byref(plan.tuning), cells.data_ptr(),
                                            cells.numel(), tr_sel.data_ptr(), s))
    est = ghost_view(plan.g, run.level(op.n_steps)[0])
    return op.grid.crop(est).clone()
