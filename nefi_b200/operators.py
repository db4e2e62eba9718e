"""B200 drop-ins for NEFI's acoustic wave operators.

:class:`WaveOperatorB200` and :class:`WaveInitialConditionOperatorB200` keep the constructor
signatures, attributes and output conventions of ``nefi.physics.wave.WaveOperator``
(nefi/physics/wave.py:582-750) and ``WaveInitialConditionOperator`` (nefi/physics/wave.py:756-872),
so ``WaveFWI.operator`` / ``Photoacoustic3D.wave_operator`` can construct them unchanged, and they
register as ``"wave_b200"`` / ``"wave_initial_condition_b200"`` for config-built use.

Forward and backward run on the GPU through ``libnefiwave.so``; the gradient is the exact discrete
adjoint of the leapfrog scheme (what torch.autograd computes through the reference's unrolled loop),
evaluated by hand-written kernels behind a ``torch.autograd.Function`` (the pattern of the
reference's ``ImplicitEulerAdjoint``, nefi/operators/pde/adjoint.py:280-330). There is no CPU path:
CPU tensors raise ``ConfigError``.
"""

from __future__ import annotations

import ctypes as C
import logging
import math
import threading
from collections.abc import Callable, Sequence

import torch
from torch.autograd.function import once_differentiable

from . import _lib
from ._compat import (
    ConfigError,
    Operator,
    OperatorError,
    ShapeError,
    SolverError,
    register,
    resample,
    shape_tuple,
)
from .geometry import (
    ABSORBING,
    GRAD_MODES,
    PaddedGrid,
    TimeAxis,
    as_points,
    damping_rate,
    pml_profile,
    ricker,
)
from .plan import DevicePlan, cached_schedule, ghost_view, plan_storage, to_ghost

log = logging.getLogger("nefi_b200")

SNAPSHOTS = ("exact", "delta16", "fixed16", "fp16", "bf16")


class _LeapfrogB200(Operator):
    """Grid, time axis and absorbing-layer bookkeeping shared by the B200 wave operators
    (the counterpart of ``_LeapfrogBase``, nefi/physics/wave.py:345-576)."""

    fidelity_tag = "wave-leapfrog"
    traceable = False

    def __init__(self, domain, receivers, *, n_t: int, dt_obs: float, c_max: float, order: int = 4,
                 absorbing: str = "pml", absorb_width: float | None = None, absorb_R: float = 1e-3,
                 cerjan_gamma: float = 0.3, courant: float = 0.9, grad_mode: str = "checkpoint",
                 checkpoint_every: int | None = None, snapshot: str = "exact",
                 memory_budget: int | None = None, checkpoint_slots: int | None = None) -> None:
        super().__init__()
        if absorbing not in ABSORBING:
            raise ConfigError(f"absorbing must be one of {ABSORBING}, got {absorbing!r}")
        if absorbing == "pml" and len(domain.shape) > 2:
            raise ConfigError("absorbing='pml' supports 1-D/2-D grids; use 'sponge' in 3-D")
        if grad_mode not in GRAD_MODES:
            raise ConfigError(f"grad_mode must be one of {GRAD_MODES}, got {grad_mode!r}")
        if n_t < 1 or dt_obs <= 0:
            raise ConfigError("n_t must be >= 1 and dt_obs > 0")
        if not 0.0 < absorb_R < 1.0:
            raise ConfigError(f"absorb_R must be in (0, 1), got {absorb_R}")
        if len(domain.shape) not in (2, 3):
            raise ConfigError("the B200 wave operators support 2-D and 3-D grids only")
        if snapshot not in SNAPSHOTS:
            raise ConfigError(f"snapshot must be one of {SNAPSHOTS}, got {snapshot!r}")
        self.domain = domain
        self.receivers = as_points(receivers, len(domain.shape), "receivers")
        self.n_t, self.dt_obs = int(n_t), float(dt_obs)
        self.c_max = float(c_max)
        self.order = int(order)
        if self.order not in (2, 4):
            raise ConfigError(f"Laplacian order must be 2 or 4, got {order}")
        self.absorbing = absorbing
        if absorb_width is None:
            absorb_width = 10.0 * max(domain.spacing()) if absorbing != "none" else 0.0
        self.absorb_width = float(absorb_width) if absorbing != "none" else 0.0
        self.absorb_R = float(absorb_R)
        self.cerjan_gamma = float(cerjan_gamma)
        self.courant = float(courant)
        self.grad_mode = grad_mode
        self.checkpoint_every = checkpoint_every
        self.snapshot = snapshot
        self.memory_budget = memory_budget
        # snapshot slots of a checkpointed gradient (None: as the memory budget allows); fewer than the
        # segments selects binomial checkpointing
        self.checkpoint_slots = checkpoint_slots
        # the wavefield storage the last gradient-carrying call chose: ("history", None),
        # ("checkpoint", segment) or ("checkpoint", segment, slots); None before the first
        self.last_storage = None
        self.grid = PaddedGrid(domain, self.absorb_width)
        ta = TimeAxis(self.n_t, self.dt_obs, self.c_max, self.grid.spacing, self.order, self.courant)
        self.substeps, self.dt, self.n_steps = ta.substeps, ta.dt, ta.n_steps
        self._plans: dict = {}
        self._res: dict = {}

    @property
    def use_pml(self) -> bool:
        return self.absorbing == "pml" and any(self.grid.n_abs)

    def _kwargs(self) -> dict:
        return {"n_t": self.n_t, "dt_obs": self.dt_obs, "c_max": self.c_max, "order": self.order,
                "absorbing": self.absorbing, "absorb_width": self.absorb_width,
                "absorb_R": self.absorb_R, "cerjan_gamma": self.cerjan_gamma,
                "courant": self.courant, "grad_mode": self.grad_mode,
                "checkpoint_every": self.checkpoint_every, "snapshot": self.snapshot,
                "memory_budget": self.memory_budget, "checkpoint_slots": self.checkpoint_slots}

    @property
    def times(self) -> torch.Tensor:
        return torch.arange(self.n_t, dtype=torch.float64) * self.dt_obs

    @property
    def record(self) -> list[int]:
        return [j * self.substeps for j in range(self.n_t)]

    def damping_profile(self) -> torch.Tensor:
        """Sponge damping rate on the padded grid (float64), as the reference defines it."""
        return damping_rate(self.grid, self.c_max, self.absorb_R)

    def pml_profile(self, ax: int, faces: bool = False) -> torch.Tensor:
        return pml_profile(self.grid, ax, self.c_max, self.absorb_R, faces)

    def _plan(self, device: torch.device, dtype: torch.dtype) -> DevicePlan:
        key = (str(device), dtype)
        if key not in self._plans:
            self._plans[key] = DevicePlan(self, device, dtype)
        return self._plans[key]

    def _check_device(self, x: torch.Tensor, name: str) -> None:
        if x.device.type != "cuda":
            raise ConfigError(f"{type(self).__name__} runs on CUDA devices only; {name} is on {x.device}")
        if x.dtype not in (torch.float32, torch.float64):
            raise ConfigError(f"{name} must be float32 or float64, got {x.dtype}")

    def _check_speed(self, c: torch.Tensor) -> None:
        lo, hi = torch.aminmax(c.detach())  # one reduction, one host round trip
        cmin, cmax = (float(v) for v in torch.stack([lo, hi]).tolist())
        if cmax > self.c_max * (1.0 + 1e-6):
            raise OperatorError(
                f"wave speed max {cmax:.4g} exceeds the c_max={self.c_max:.4g} used for the CFL "
                "time step; raise c_max or bound the field (e.g. a Bounded head)")
        if cmin <= 0:
            raise OperatorError("wave speed must be positive everywhere")

    def _budget(self, device: torch.device) -> int:
        if self.memory_budget is not None:
            return int(self.memory_budget)
        # memory the driver has free plus blocks PyTorch's caching allocator holds unused (the last
        # gradient's history, say): the allocator hands those out again, or frees them on a miss
        free, _ = torch.cuda.mem_get_info(device)
        idle = torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
        return int(0.85 * (free + max(idle, 0)))

    def extra_repr(self) -> str:
        g = self.grid
        return (f"shape={g.shape}, padded={g.padded_shape}, n_t={self.n_t}, dt_obs={self.dt_obs:.4g}, "
                f"dt={self.dt:.4g} (x{self.substeps}), order={self.order}, absorbing={self.absorbing}")


# ------------------------------------------------------------------------------------------------
# shared sweep helpers
# ------------------------------------------------------------------------------------------------
class _Run:
    """Buffers of one forward sweep that the backward sweep needs."""

    def __init__(self, plan: DevicePlan, n_shots: int, n_steps: int, mode, snapshot: str):
        self.plan, self.n_shots = plan, n_shots
        self.kind = mode[0]
        self.storage = _lib.Storage()
        self.history = self.ring = self.snap = self.segbuf = None
        # the pressure advances through three rotating levels in every mode (four when the forward
        # takes two steps per launch)
        self.nl = plan.ring_levels
        self.ring = plan.empty_levels(self.nl, n_shots)
        self.storage.ring = self.ring.data_ptr()
        self.storage.ring_levels = self.nl
        self.psi = None
        if plan.pml is not None:  # the PML's face fields, two axes x two step parities, zero at start
            self.psi = plan.empty_levels(4, n_shots)
            self.storage.pml_psi = self.psi.data_ptr()
        if self.kind == "history":
            # step n stores Lap p^n into the interior of level n; nothing reads the ghost cells
            # (the adjoint multiplies them only into sums of cells outside the grid, never stored)
            self.history = plan.empty_levels(n_steps, n_shots, zero=False)
            self.storage.history = self.history.data_ptr()
        elif self.kind == "checkpoint":
            k = int(mode[1])
            kind = _lib.SNAP_KINDS[snapshot]
            n_snap = -(-n_steps // k) if n_steps > 0 else 1
            self.schedule = None
            if len(mode) > 2 and mode[2] < n_snap:  # binomial checkpointing over mode[2] slots
                sweep_slot, program = cached_schedule(n_snap, int(mode[2]))
                self.schedule = (sweep_slot, program)  # host arrays the library reads during the calls
                self.storage.snap_slot = sweep_slot.data_ptr()
                self.storage.schedule = program.data_ptr()
                self.storage.n_schedule = program.numel() // 3
                n_snap = int(mode[2])
            nbytes = plan.snapshot_bytes(n_shots, n_snap, kind)
            self.snap = torch.empty(nbytes, dtype=torch.uint8, device=plan.device)
            self.segbuf = plan.empty_levels(k, n_shots)
            self.storage.snap = self.snap.data_ptr()
            self.storage.segbuf = self.segbuf.data_ptr()
            self.storage.segment = k
            self.storage.snap_kind = kind

    def level(self, n: int) -> torch.Tensor:
        """Pressure level ``n`` (``(n_shots, field)``) while it is in the ring."""
        return self.ring[(n + 1) % self.nl]

    def release(self) -> None:
        self.history = self.ring = self.snap = self.segbuf = self.psi = None


def _forward_sweep(plan: DevicePlan, medium, acq, run: _Run, n_begin: int, n_end: int,
                   traces: torch.Tensor | None, stream: int) -> None:
    lib = _lib.load()
    _lib.check(lib.nw_forward(C.byref(plan.g), C.byref(medium), C.byref(acq), C.byref(plan.time),
                              C.byref(run.storage), C.byref(plan.tuning), n_begin, n_end,
                              _lib.ptr(traces), stream))


def _adjoint_sweep(plan: DevicePlan, medium, acq, run: _Run, grad_traces: torch.Tensor,
                   want_initial: bool, stream: int):
    lib = _lib.load()
    S = run.n_shots
    work = plan.empty_levels(7 if plan.pml is not None else 3, S, zero=False)
    gC = torch.empty(plan.n_acc(S), plan.field, device=plan.device, dtype=plan.dtype)
    lam0 = mu1 = None
    if want_initial:
        lam0 = plan.empty_levels(1, S, zero=False)[0]
        mu1 = plan.empty_levels(1, S, zero=False)[0]
    _lib.check(lib.nw_adjoint(C.byref(plan.g), C.byref(medium), C.byref(acq), C.byref(plan.time),
                              C.byref(run.storage), C.byref(plan.tuning), grad_traces.data_ptr(),
                              work.data_ptr(), gC.data_ptr(), _lib.ptr(lam0), _lib.ptr(mu1), stream))
    if run.storage.snap and run.storage.snap_kind != _lib.NW_SNAP_EXACT:
        # encoded snapshots carry a validity check; reading the status synchronises the stream, which
        # a graph capture cannot do: there the graph reads it after each replay
        if torch.cuda.is_current_stream_capturing():
            _deferred_status.pending = True
        else:
            _check_snapshot_status(stream)
    return gC, lam0, mu1


class _Deferred(threading.local):
    pending = False


_deferred_status = _Deferred()  # set while a capture records an adjoint that decodes snapshots


def _check_snapshot_status(stream: int) -> None:
    """Synchronise ``stream`` and raise if a snapshot decode found a non-finite value."""
    rc = _lib.load().nw_status(stream)
    if rc == _lib.NW_ERR_NONFINITE:
        raise SolverError("a wavefield snapshot held a non-finite value: the forward run diverged "
                          "or the snapshot pool was corrupted")
    _lib.check(rc)


# ------------------------------------------------------------------------------------------------
# FWI
# ------------------------------------------------------------------------------------------------
class _FWIFunction(torch.autograd.Function):
    @staticmethod
    @_lib.on_device
    def forward(ctx, c: torch.Tensor, op: "WaveOperatorB200", shot0: int, n_shots: int):
        plan = op._plan(c.device, c.dtype)
        stream = _lib.stream_handle(c.device)
        lib = _lib.load()
        c = c.contiguous()
        c2dt2 = torch.empty(plan.field, device=c.device, dtype=c.dtype)
        _lib.check(lib.nw_prepare_medium(C.byref(plan.g), plan.n_abs, c.data_ptr(), op.dt**2,
                                         c2dt2.data_ptr(), stream))
        medium = plan.medium(c2dt2)
        acq = plan.acquisition(n_shots, shot0)
        needs_grad = ctx.needs_input_grad[0]
        mode = (plan_storage(plan, n_shots, op.n_steps, op.grad_mode, op.checkpoint_every,
                             op.snapshot, op._budget(c.device), op.checkpoint_slots) if needs_grad else ("ring", None))
        op.last_storage = tuple(mode)
        run = _Run(plan, n_shots, op.n_steps, mode, op.snapshot)
        traces = torch.empty(n_shots, plan.n_rec, op.n_t, device=c.device, dtype=c.dtype)
        _forward_sweep(plan, medium, acq, run, 0, op.n_steps, traces, stream)
        if needs_grad:
            ctx.op, ctx.run, ctx.shot0, ctx.n_shots = op, run, shot0, n_shots
            ctx.c2dt2 = c2dt2
            ctx.save_for_backward(c)
        else:
            run.release()
        return traces

    @staticmethod
    @once_differentiable
    @_lib.on_device
    def backward(ctx, grad_traces: torch.Tensor):
        (c,) = ctx.saved_tensors
        op, run = ctx.op, ctx.run
        plan = run.plan
        stream = _lib.stream_handle(c.device)
        medium = plan.medium(ctx.c2dt2)
        acq = plan.acquisition(ctx.n_shots, ctx.shot0)
        gtr = grad_traces.contiguous().to(c.dtype)
        gC, _, _ = _adjoint_sweep(plan, medium, acq, run, gtr, False, stream)
        grad64 = torch.empty(c.shape, device=c.device, dtype=torch.float64)
        _lib.check(_lib.load().nw_reduce_grad_c(C.byref(plan.g), plan.n_abs, c.data_ptr(), op.dt**2,
                                                gC.shape[0], gC.data_ptr(), 0, grad64.data_ptr(),
                                                stream))
        run.release()
        ctx.run = None
        return grad64.to(c.dtype), None, None, None


@register("operator", "wave_b200")
class WaveOperatorB200(_LeapfrogB200):
    """Acoustic FWI forward model on the B200: sound speed ``c(x)`` -> traces of every source.

    Same arguments as ``nefi.physics.wave.WaveOperator`` (nefi/physics/wave.py:610-632), plus
    ``snapshot`` (encoding of checkpoint snapshots: ``"exact"``; ``"delta16"``, int16 second
    differences in time with per-block scales, whose float32 gradient stays within 1e-4 of float64;
    ``"fixed16"``, ``"fp16"`` and ``"bf16"``, block-scaled 16-bit values that do not meet that bound:
    1.8e-4, 2.0e-3 and 1.7e-2 on a 128^2, 1000-step case) and ``memory_budget`` (bytes available for
    wavefield storage; default 85 % of the device memory that is free or held unused by PyTorch's
    allocator).
    Output ``(n_sources, n_receivers, n_t)`` at ``t_j = j dt_obs``; the gradient w.r.t. ``c`` is
    the exact discrete adjoint, reduced over shots in float64.
    """

    def __init__(self, domain, sources, receivers, *, n_t: int, dt_obs: float, f0: float,
                 c_max: float, field: str = "c", t0: float | None = None, amplitude: float = 1.0,
                 order: int = 4, absorbing: str = "pml", absorb_width: float | None = None,
                 absorb_R: float = 1e-3, cerjan_gamma: float = 0.3, courant: float = 0.9,
                 grad_mode: str = "checkpoint", checkpoint_every: int | None = None,
                 source_batch: int | None = None, snapshot: str = "exact",
                 memory_budget: int | None = None, checkpoint_slots: int | None = None) -> None:
        super().__init__(domain, receivers, n_t=n_t, dt_obs=dt_obs, c_max=c_max, order=order,
                         absorbing=absorbing, absorb_width=absorb_width, absorb_R=absorb_R,
                         cerjan_gamma=cerjan_gamma, courant=courant, grad_mode=grad_mode,
                         checkpoint_every=checkpoint_every, snapshot=snapshot,
                         memory_budget=memory_budget, checkpoint_slots=checkpoint_slots)
        self.primary = field
        self.homogeneity = None
        self.sources = as_points(sources, len(domain.shape), "sources")
        self.f0 = float(f0)
        self.t0 = 1.2 / self.f0 if t0 is None else float(t0)
        self.amplitude = float(amplitude)
        self.source_batch = source_batch
        self.fidelity_tag = f"wave-leapfrog-o{self.order}-{self.absorbing}"
        # validate the acquisition on the host now (ConfigError for points outside the grid)
        self.grid.point_stencils(self.sources)
        self.grid.point_stencils(self.receivers)

    @property
    def n_sources(self) -> int:
        return int(self.sources.shape[0])

    @property
    def n_receivers(self) -> int:
        return int(self.receivers.shape[0])

    def wavelet(self) -> torch.Tensor:
        t = torch.arange(self.n_steps, dtype=torch.float64) * self.dt
        return self.amplitude * ricker(t, self.f0, self.t0)

    def at_resolution(self, shape):
        shape = shape_tuple(shape)
        if shape == tuple(self.domain.shape):
            return self
        if shape not in self._res:
            op = WaveOperatorB200(self.domain.at(shape), self.sources, self.receivers, f0=self.f0,
                                  t0=self.t0, amplitude=self.amplitude, field=self.primary,
                                  source_batch=self.source_batch, **self._kwargs())
            op.fidelity_tag = self.fidelity_tag
            self._res[shape] = op
        return self._res[shape]

    def output_shape(self, shape):
        return (self.n_sources, self.n_receivers, self.n_t)

    def _validate(self, c: torch.Tensor) -> None:
        if tuple(c.shape) != tuple(self.domain.shape):
            raise ShapeError(f"c has shape {tuple(c.shape)}, operator expects {self.domain.shape}")
        self._check_device(c, "c")
        self._check_speed(c)

    def forward(self, fields) -> torch.Tensor:
        c = self.get_field(fields)
        self._validate(c)
        n = self.n_sources
        chunk = self.source_batch or n
        outs = [_FWIFunction.apply(c, self, s0, min(n, s0 + chunk) - s0) for s0 in range(0, n, chunk)]
        return outs[0] if len(outs) == 1 else torch.cat(outs, dim=0)

    @_lib.on_device
    def misfit_gradient(self, c: torch.Tensor, observed: torch.Tensor, events: dict | None = None,
                        misfit=None, mask: torch.Tensor | None = None):
        """One FWI gradient without autograd: ``(J, dJ/dc)`` for ``J = 1/2 ||F(c) - observed||^2``, or,
        given a :class:`nefi_b200.misfit.TraceMisfit` ``misfit``, for its band-limited (relative) MSE
        with observation weights ``mask``; that loss and its adjoint source come from one fused pass
        over each chunk's traces.

        ``dJ/dc`` is returned in float64 (the cross-shot reduction is float64), ready for a
        cross-device sum. All shots run in one sweep (``source_batch`` chunks them when set).
        ``events``, if given, receives CUDA events ``fwd0, fwd1, adj0, adj1`` recorded on the
        current stream around the forward and adjoint sweeps of the first chunk.
        """
        self._validate(c)
        if tuple(observed.shape) != (self.n_sources, self.n_receivers, self.n_t):
            raise ShapeError(f"observed has shape {tuple(observed.shape)}, expected "
                             f"{(self.n_sources, self.n_receivers, self.n_t)}")
        return self._gradient(c, observed, events, misfit, mask, self._storage_modes(c))

    def _storage_modes(self, c: torch.Tensor) -> list:
        """Wavefield storage of each source chunk of a gradient (host decision, no device work)."""
        plan = self._plan(c.device, c.dtype)
        n = self.n_sources
        chunk = self.source_batch or n
        budget = self._budget(c.device)
        return [plan_storage(plan, min(n, s0 + chunk) - s0, self.n_steps, self.grad_mode, self.checkpoint_every,
                             self.snapshot, budget, self.checkpoint_slots) for s0 in range(0, n, chunk)]

    def _gradient(self, c, observed, events, misfit, mask, modes):
        """The device work of ``misfit_gradient`` (validated inputs, storage decided): enqueues only,
        with no host synchronisation, so that it can be recorded in a CUDA graph."""
        plan = self._plan(c.device, c.dtype)
        stream = _lib.stream_handle(c.device)
        lib = _lib.load()
        # timing events recorded inside a graph capture must become event-record nodes of the graph
        ext = torch.cuda.is_current_stream_capturing()
        c = c.detach().contiguous()
        c2dt2 = torch.empty(plan.field, device=c.device, dtype=c.dtype)
        _lib.check(lib.nw_prepare_medium(C.byref(plan.g), plan.n_abs, c.data_ptr(), self.dt**2,
                                         c2dt2.data_ptr(), stream))
        medium = plan.medium(c2dt2)
        grad = torch.zeros(c.shape, device=c.device, dtype=torch.float64)
        loss = torch.zeros((), device=c.device, dtype=torch.float64)
        if misfit is not None:
            misfit.prepare(observed.to(c.dtype), mask)
        n = self.n_sources
        chunk = self.source_batch or n
        for k, s0 in enumerate(range(0, n, chunk)):
            S = min(n, s0 + chunk) - s0
            acq = plan.acquisition(S, s0)
            mode = modes[k]
            self.last_storage = tuple(mode)
            tm = events if (events is not None and s0 == 0) else None
            run = _Run(plan, S, self.n_steps, mode, self.snapshot)
            traces = torch.empty(S, plan.n_rec, self.n_t, device=c.device, dtype=c.dtype)
            if tm is not None:
                tm["fwd0"] = torch.cuda.Event(enable_timing=True, external=ext)
                tm["fwd0"].record()
            _forward_sweep(plan, medium, acq, run, 0, self.n_steps, traces, stream)
            if tm is not None:
                tm["fwd1"] = torch.cuda.Event(enable_timing=True, external=ext)
                tm["fwd1"].record()
            if misfit is None:
                resid = traces - observed[s0:s0 + S].to(c.dtype)
                loss += 0.5 * resid.double().square().sum()
            else:
                j, resid = misfit.value_and_grad(traces, rows=slice(s0, s0 + S))
            if tm is not None:
                tm["adj0"] = torch.cuda.Event(enable_timing=True, external=ext)
                tm["adj0"].record()
            gC, _, _ = _adjoint_sweep(plan, medium, acq, run, resid.contiguous(), False, stream)
            _lib.check(lib.nw_reduce_grad_c(C.byref(plan.g), plan.n_abs, c.data_ptr(), self.dt**2,
                                            gC.shape[0], gC.data_ptr(), 1, grad.data_ptr(), stream))
            if tm is not None:
                tm["adj1"] = torch.cuda.Event(enable_timing=True, external=ext)
                tm["adj1"].record()
            run.release()
        if misfit is not None:
            loss = j.clone()
        return loss, grad

    FWD_CANDIDATES = ((4, 2, 2, 1), (4, 2, 1, 1), (2, 4, 2, 1), (4, 4, 2, 1), (4, 4, 2, 2), (4, 2, 2, 2))
    ADJ_CANDIDATES = ((2, 2, 4), (2, 2, 8), (2, 4, 4), (2, 2, 2))

    @_lib.on_device
    def autotune(self, c: torch.Tensor, steps: int = 200, fwd_candidates=None, adj_candidates=None,
                 repeats: int = 2) -> tuple:
        """Choose this operator's 2-D launch shapes and forward steps per launch by timing candidates
        on the device (CUDA events around the sweeps of graph-replayed gradients), on a copy of the
        operator shortened to about ``steps`` leapfrog steps (the per-step cost does not depend on the
        step count). The forward candidates ``(vz, rx,
        shots_per_cta, depth)`` are timed with the default adjoint shape, then the adjoint candidates
        ``(vz, rx, shots_per_cta)`` with the forward chosen; depth 2 (two steps per launch) applies to
        2-D grids without a PML and falls back to one step elsewhere. Candidates the library refuses
        (a shape above the shared-memory limit, a float64 tile of four columns per thread) are
        skipped. Sets ``self.tuning`` and returns it; ``self.autotune_results`` holds the microseconds
        per step of each candidate. Traces are bitwise the same under every tuning; the gradient
        regroups its float sums with the adjoint's shots per CTA."""
        self._validate(c)
        if len(self.domain.shape) != 2:
            return getattr(self, "tuning", None)
        n_t = max(2, min(self.n_t, steps // self.substeps + 1))
        short = WaveOperatorB200(self.domain, self.sources, self.receivers, f0=self.f0, t0=self.t0,
                                 amplitude=self.amplitude, **{**self._kwargs(), "n_t": n_t})
        short.source_batch = self.source_batch
        obs = torch.zeros(short.n_sources, short.n_receivers, short.n_t, device=c.device, dtype=c.dtype)
        results = {}

        def per_step(tuning):  # (forward, adjoint) microseconds per step, best of `repeats`
            # timed as graph replays, the way the gradient graphs and the batches run: eager sweeps
            # add the host's launch time per step, which differs between the layers (the PML's
            # side stream) and can rank the candidates differently
            short.tuning = tuning
            short._plans.clear()
            fwd = adj = math.inf
            try:
                short.misfit_gradient(c, obs)  # a shape the library refuses raises here, not in a capture
                g = short.gradient_graph(c, obs, events=True)
            except _lib.LibraryError:
                return math.inf, math.inf
            for r in range(repeats + 1):
                g.replay()
                torch.cuda.synchronize(c.device)
                if r:
                    ev = g.events
                    fwd = min(fwd, ev["fwd0"].elapsed_time(ev["fwd1"]) * 1e3 / short.n_steps)
                    adj = min(adj, ev["adj0"].elapsed_time(ev["adj1"]) * 1e3 / short.n_steps)
            g.check()
            g.release()
            del g
            results[tuning] = (fwd, adj)
            return fwd, adj

        fwd_c = fwd_candidates or self.FWD_CANDIDATES
        adj_c = adj_candidates or self.ADJ_CANDIDATES
        best_f = min(fwd_c, key=lambda f: per_step((*f[:3], 0, 0, 0, f[3]))[0])
        best_a = min(adj_c, key=lambda a: per_step((*best_f[:3], *a, best_f[3]))[1])
        if math.isinf(results.get((*best_f[:3], *best_a, best_f[3]), (math.inf, math.inf))[1]):
            raise ConfigError("autotune: the library refused every candidate launch shape")
        self.tuning = (*best_f[:3], *best_a, best_f[3])
        self._plans.clear()
        self.autotune_results = results
        return self.tuning

    @_lib.on_device
    def gradient_graph(self, c: torch.Tensor, observed: torch.Tensor, events: bool = False) -> "GradientGraph":
        """``misfit_gradient(c, observed)`` recorded once as a CUDA graph: a :class:`GradientGraph` whose
        ``replay()`` recomputes ``loss`` and ``grad`` from its static inputs ``c`` and ``observed``
        (copies of the arguments; write new values into them with ``run``). The speed check of
        ``c`` and the storage decision are made when the graph is recorded and by ``run``, not by
        ``replay``. ``events=True`` also records timing events around the first chunk's forward and
        adjoint sweeps (``GradientGraph.events``)."""
        self._validate(c)
        if tuple(observed.shape) != (self.n_sources, self.n_receivers, self.n_t):
            raise ShapeError(f"observed has shape {tuple(observed.shape)}, expected "
                             f"{(self.n_sources, self.n_receivers, self.n_t)}")
        return GradientGraph(self, c, observed, events)

    @_lib.on_device
    def simulate(self, c: torch.Tensor, observe: Callable | None = None,
                 record: Sequence[int] | None = None, sources: slice | None = None):
        """Leapfrog run returning ``(state, obs)`` like the reference's ``simulate``
        (nefi/physics/wave.py:699-740).

        Without ``observe`` the receiver samples at the record steps are returned. With
        ``observe(state, n)`` the run advances one launch at a time and hands ``observe`` the
        padded state ``(p^{n-1}, p^n)`` (views of device memory) at every ``n`` in ``record``
        (default every step): a debugging path, not the fast one. No gradient flows here.
        """
        self._validate(c)
        plan = self._plan(c.device, c.dtype)
        sl = sources or slice(0, self.n_sources)
        shot0, stop, _ = sl.indices(self.n_sources)
        S = stop - shot0
        stream = _lib.stream_handle(c.device)
        lib = _lib.load()
        c2dt2 = torch.empty(plan.field, device=c.device, dtype=c.dtype)
        _lib.check(lib.nw_prepare_medium(C.byref(plan.g), plan.n_abs, c.detach().contiguous().data_ptr(),
                                         self.dt**2, c2dt2.data_ptr(), stream))
        medium, acq = plan.medium(c2dt2), plan.acquisition(S, shot0)
        run = _Run(plan, S, self.n_steps, ("ring", None), self.snapshot)
        if observe is None:
            traces = torch.empty(S, plan.n_rec, self.n_t, device=c.device, dtype=c.dtype)
            _forward_sweep(plan, medium, acq, run, 0, self.n_steps, traces, stream)
            state = tuple(ghost_view(plan.g, run.level(n)) for n in (self.n_steps - 1, self.n_steps))
            return state, list(traces.unbind(-1))
        rec = set(range(1, self.n_steps + 1)) if record is None else {int(n) for n in record}
        obs = []

        def _obs(n):
            if n in rec:
                o = observe(tuple(ghost_view(plan.g, run.level(m)) for m in (n - 1, n)), n)
                if o is not None:
                    obs.append(o)

        _obs(0)
        for n in range(self.n_steps):
            _forward_sweep(plan, medium, acq, run, n, n + 1, None, stream)
            _obs(n + 1)
        state = tuple(ghost_view(plan.g, run.level(n)).clone() for n in (self.n_steps - 1, self.n_steps))
        return state, obs


# ------------------------------------------------------------------------------------------------
# photoacoustic (initial value)
# ------------------------------------------------------------------------------------------------
class _PATFunction(torch.autograd.Function):
    @staticmethod
    @_lib.on_device
    def forward(ctx, p0: torch.Tensor, c: torch.Tensor, op: "WaveInitialConditionOperatorB200",
                c2dt2_known: torch.Tensor | None):
        plan = op._plan(p0.device, p0.dtype)
        stream = _lib.stream_handle(p0.device)
        lib = _lib.load()
        d = plan.pgrid.d
        batch = tuple(p0.shape[: p0.ndim - d])
        S = int(math.prod(batch)) if batch else 1
        p0f = p0.detach().reshape(S, *plan.pgrid.shape).contiguous()
        if c2dt2_known is not None:  # the fixed medium, formed once in float64 on the host
            c2dt2 = c2dt2_known
        else:
            c2dt2 = torch.empty(plan.field, device=p0.device, dtype=p0.dtype)
            _lib.check(lib.nw_prepare_medium(C.byref(plan.g), plan.n_abs, c.detach().contiguous().data_ptr(),
                                             op.dt**2, c2dt2.data_ptr(), stream))
        medium = plan.medium(c2dt2)
        acq = plan.acquisition(S)
        need_p0, need_c = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        needs_grad = need_p0 or need_c
        mode = (plan_storage(plan, S, op.n_steps, op.grad_mode, op.checkpoint_every, op.snapshot,
                             op._budget(p0.device), op.checkpoint_slots) if needs_grad else ("ring", None))
        run = _Run(plan, S, op.n_steps, mode, op.snapshot)
        _lib.check(lib.nw_initial_state(C.byref(plan.g), plan.n_abs, C.byref(medium), S, p0f.data_ptr(),
                                        run.level(-1).data_ptr(), run.level(0).data_ptr(), stream))
        p0_level = run.level(0).clone() if need_c else None
        traces = torch.empty(S, plan.n_rec, op.n_t, device=p0.device, dtype=p0.dtype)
        _forward_sweep(plan, medium, acq, run, 0, op.n_steps, traces, stream)
        if needs_grad:
            ctx.op, ctx.run, ctx.S, ctx.batch, ctx.c2dt2, ctx.p0_level = op, run, S, batch, c2dt2, p0_level
            ctx.save_for_backward(c)
        else:
            run.release()
        return traces.reshape(*batch, plan.n_rec, op.n_t)

    @staticmethod
    @once_differentiable
    @_lib.on_device
    def backward(ctx, grad_traces: torch.Tensor):
        (c,) = ctx.saved_tensors
        op, run, S = ctx.op, ctx.run, ctx.S
        plan = run.plan
        dev = grad_traces.device
        stream = _lib.stream_handle(dev)
        lib = _lib.load()
        medium = plan.medium(ctx.c2dt2)
        acq = plan.acquisition(S)
        gtr = grad_traces.reshape(S, plan.n_rec, op.n_t).contiguous().to(plan.dtype)
        gC, lam0, mu1 = _adjoint_sweep(plan, medium, acq, run, gtr, True, stream)
        need_c = ctx.needs_input_grad[1]
        grad_p0 = torch.empty(S, *plan.pgrid.shape, device=dev, dtype=plan.dtype)
        p0l = ctx.p0_level if need_c else lam0
        _lib.check(lib.nw_initial_state_adjoint(C.byref(plan.g), plan.n_abs, C.byref(medium),
                                                C.byref(plan.time), S, lam0.data_ptr(), mu1.data_ptr(),
                                                p0l.data_ptr(), grad_p0.data_ptr(),
                                                gC.data_ptr() if need_c else None, plan.shots_per_acc(S),
                                                stream))
        grad_c = None
        if need_c:
            g64 = torch.empty(c.shape, device=dev, dtype=torch.float64)
            _lib.check(lib.nw_reduce_grad_c(C.byref(plan.g), plan.n_abs, c.contiguous().data_ptr(),
                                            op.dt**2, gC.shape[0], gC.data_ptr(), 0, g64.data_ptr(), stream))
            grad_c = g64.to(c.dtype)
        run.release()
        ctx.run = None
        ctx.p0_level = None
        gp0 = grad_p0.reshape(*ctx.batch, *plan.pgrid.shape) if ctx.needs_input_grad[0] else None
        return gp0, grad_c, None, None


class GradientGraph:
    """One FWI gradient of a :class:`WaveOperatorB200` recorded as a CUDA graph (see
    ``WaveOperatorB200.gradient_graph``). The graph owns its wavefield storage for its lifetime."""

    def __init__(self, op: "WaveOperatorB200", c: torch.Tensor, observed: torch.Tensor, events: bool):
        self.op = op
        self.device = c.device
        self.c = c.detach().contiguous().clone()
        self.observed = observed.to(c.dtype).contiguous().clone()
        self._modes = op._storage_modes(self.c)
        lib = _lib.load()
        op._gradient(self.c, self.observed, None, None, None, self._modes)  # kernels loaded, opt-ins done
        torch.cuda.synchronize(self.device)
        self.events = {} if events else None
        graph = torch.cuda.CUDAGraph()
        n0 = lib.nw_launch_count()
        _deferred_status.pending = False
        try:
            with torch.cuda.graph(graph):
                self.loss, self.grad = op._gradient(self.c, self.observed, self.events, None, None, self._modes)
        finally:
            # the adjoint decodes encoded snapshots: their status is read after each replay instead
            self.checks_status = _deferred_status.pending
            _deferred_status.pending = False
        self.launches = int(lib.nw_launch_count() - n0)  # this library's kernels per replay
        self._graph = graph
        torch.cuda.synchronize(self.device)

    def replay(self) -> None:
        """Recompute ``loss`` and ``grad`` from the current ``c`` and ``observed`` (asynchronous; with
        encoded snapshots, ``check()`` afterwards raises if a decode met a non-finite value)."""
        self._graph.replay()

    def check(self) -> None:
        """Synchronise and raise ``SolverError`` if a snapshot decode of the replays since the last
        check met a non-finite value (no-op without encoded snapshots)."""
        if self.checks_status:
            _check_snapshot_status(_lib.stream_handle(self.device))

    def run(self, c: torch.Tensor, observed: torch.Tensor):
        """Check ``c`` like the operator does, copy both inputs in, replay and (with encoded snapshots)
        check their status; returns ``(loss, grad)``."""
        self.op._validate(c)
        self.c.copy_(c)
        self.observed.copy_(observed)
        self.replay()
        self.check()
        return self.loss, self.grad

    def release(self) -> None:
        self._graph = None
        self.loss = self.grad = None


@register("operator", "wave_initial_condition_b200")
class WaveInitialConditionOperatorB200(_LeapfrogB200):
    """Photoacoustic forward model on the B200: initial pressure ``p0`` -> traces.

    Same arguments as ``nefi.physics.wave.WaveInitialConditionOperator``
    (nefi/physics/wave.py:769-787) plus ``snapshot`` and ``memory_budget`` (as for
    :class:`WaveOperatorB200`: only ``"exact"`` and ``"delta16"`` snapshots keep the float32 gradient
    within 1e-4 of float64). Linear in ``p0``
    (``homogeneity = 1``); leading batch dims of ``p0`` are kept. The known sound speed ``c`` is a
    buffer as in the reference; :meth:`with_speed` evaluates the operator for a differentiable
    sound-speed map, giving the gradient w.r.t. ``c`` as well.
    """

    def __init__(self, domain, receivers, *, n_t: int, dt_obs: float, c=1.0, c_max: float | None = None,
                 field: str = "p0", order: int = 4, absorbing: str = "pml",
                 absorb_width: float | None = None, absorb_R: float = 1e-3, cerjan_gamma: float = 0.3,
                 courant: float = 0.9, grad_mode: str = "checkpoint", checkpoint_every: int | None = None,
                 snapshot: str = "exact", memory_budget: int | None = None,
                 checkpoint_slots: int | None = None) -> None:
        c_t = torch.as_tensor(c, dtype=torch.float64)
        if c_t.ndim not in (0, len(domain.shape)):
            raise ShapeError("c must be a scalar or a map on the domain grid")
        if c_t.ndim > 0 and tuple(c_t.shape) != tuple(domain.shape):
            c_t = resample(c_t, domain.shape)
        c_max = float(c_t.max()) if c_max is None else float(c_max)
        super().__init__(domain, receivers, n_t=n_t, dt_obs=dt_obs, c_max=c_max, order=order,
                         absorbing=absorbing, absorb_width=absorb_width, absorb_R=absorb_R,
                         cerjan_gamma=cerjan_gamma, courant=courant, grad_mode=grad_mode,
                         checkpoint_every=checkpoint_every, snapshot=snapshot,
                         memory_budget=memory_budget, checkpoint_slots=checkpoint_slots)
        self.primary = field
        self.homogeneity = 1.0
        self.c_known = c_t
        self.fidelity_tag = f"wave-leapfrog-ic-o{self.order}-{self.absorbing}"
        self.grid.point_stencils(self.receivers)
        self._c_dev: dict = {}

    def at_resolution(self, shape):
        shape = shape_tuple(shape)
        if shape == tuple(self.domain.shape):
            return self
        if shape not in self._res:
            c = self.c_known
            if c.ndim > 0:
                c = resample(c, shape)
            op = WaveInitialConditionOperatorB200(self.domain.at(shape), self.receivers, c=c,
                                                  field=self.primary, **self._kwargs())
            op.fidelity_tag = self.fidelity_tag
            self._res[shape] = op
        return self._res[shape]

    def output_shape(self, shape):
        return (int(self.receivers.shape[0]), self.n_t)

    def _known_speed(self, device, dtype) -> tuple[torch.Tensor, torch.Tensor]:
        """The fixed sound speed and its ``c^2 dt^2`` in the ghost layout. Like the reference
        (nefi/physics/wave.py:814-820) the product is formed in float64 and then cast."""
        key = (str(device), dtype)
        if key not in self._c_dev:
            c = self.c_known
            if c.ndim == 0:
                c = c.expand(self.domain.shape)
            plan = self._plan(device, dtype)
            c2 = (self.grid.pad(c.to(torch.float64), "replicate") ** 2 * self.dt**2).to(dtype)
            self._c_dev[key] = (c.to(dtype).contiguous().to(device), to_ghost(plan.g, c2).to(device))
        return self._c_dev[key]

    def _validate(self, p0: torch.Tensor) -> None:
        d = len(self.domain.shape)
        if tuple(p0.shape[p0.ndim - d:]) != tuple(self.domain.shape):
            raise ShapeError(f"p0 has shape {tuple(p0.shape)}, operator expects (..., {self.domain.shape})")
        self._check_device(p0, "p0")

    def forward(self, fields) -> torch.Tensor:
        p0 = self.get_field(fields)
        self._validate(p0)
        c, c2dt2 = self._known_speed(p0.device, p0.dtype)
        return _PATFunction.apply(p0, c, self, c2dt2)

    def with_speed(self, p0: torch.Tensor, c: torch.Tensor) -> torch.Tensor:
        """Traces for initial pressure ``p0`` in sound speed ``c`` (domain grid), differentiable
        in both. ``c`` must stay below ``c_max``, which fixed the time step."""
        self._validate(p0)
        if tuple(c.shape) != tuple(self.domain.shape):
            raise ShapeError(f"c has shape {tuple(c.shape)}, operator expects {self.domain.shape}")
        self._check_device(c, "c")
        self._check_speed(c)
        return _PATFunction.apply(p0, c.to(p0.dtype), self, None)
