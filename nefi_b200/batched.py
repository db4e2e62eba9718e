"""Many independent 2-D FWI problems in one batched sweep (``nw_batch_*``).

The reference cannot batch wave operators (nefi/solve/batched.py:68-77): each problem runs its own
time loop. Here a batch of problems with different grids, shot counts and step counts advances
together, one kernel launch per time step for all problems still running (the problems are ordered
by step count, so those are a prefix of the batch table). Storage is checkpointed with one segment
length for the batch (16-bit snapshots by default); the adjoint recomputes each segment for all
problems at once. ``BatchedFWI.capture()`` records the whole gradient (forward sweep, misfit,
adjoint sweep, float64 reductions) as one CUDA graph that ``misfit_gradients`` then replays;
``autotune()`` picks
the tile shapes of the forward and adjoint steps by timing candidates on a shortened batch.

Each problem's traces and gradient equal what ``WaveOperatorB200.misfit_gradient`` gives it alone
with the same tuning, segment length and snapshot kind (the same kernels, bitwise).
"""

from __future__ import annotations

import ctypes as C
import math
from collections.abc import Sequence

import torch

from . import _lib
from ._compat import ConfigError
from .operators import WaveOperatorB200


class BatchedFWI:
    """Misfit gradients ``J_i = 1/2 ||F_i(c_i) - d_i||^2`` of a batch of FWI operators, or with
    ``misfits`` (one :class:`nefi_b200.misfit.TraceMisfit` per operator, optional ``masks``) their
    band-limited (relative) MSE, loss and adjoint source from the fused misfit pass."""

    def __init__(self, ops: Sequence[WaveOperatorB200], *, device: torch.device | str = "cuda",
                 dtype: torch.dtype = torch.float32, segment: int | None = None, snapshot: str = "delta16",
                 tuning: Sequence[int] | None = None, misfits: Sequence | None = None,
                 masks: Sequence | None = None) -> None:
        if not ops:
            raise ConfigError("an empty batch")
        for op in ops:
            if not isinstance(op, WaveOperatorB200) or len(op.domain.shape) != 2:
                raise ConfigError("BatchedFWI takes 2-D WaveOperatorB200 problems")
            if op.order != ops[0].order:
                raise ConfigError("the problems of a batch share one stencil order")
        self.device = torch.device(device)
        self.dtype = dtype
        self.ops = list(ops)
        # table order: non-increasing step count (the active problems of a step are a prefix)
        self.order = sorted(range(len(ops)), key=lambda i: -ops[i].n_steps)
        n_max = max(op.n_steps for op in ops)
        self.segment = int(segment) if segment else max(1, int(math.ceil(math.sqrt(max(1, n_max)))))
        self.snapshot = snapshot
        self.tuning = tuple(tuning)[:6] if tuning else (0, 0, 0, 0, 0, 0)  # one step per launch
        if misfits is not None and len(misfits) != len(ops):
            raise ConfigError("misfits: one per operator")
        if masks is not None and (misfits is None or len(masks) != len(ops)):
            raise ConfigError("masks: one per operator, with misfits")
        self.misfits = list(misfits) if misfits is not None else None
        self.masks = list(masks) if masks is not None else [None] * len(ops)
        self._graph = None
        self._build()

    # -- buffers and the device table ----------------------------------------------------------
    @_lib.on_device
    def _build(self) -> None:
        lib = _lib.load()
        dev, K = self.device, self.segment
        kind = _lib.SNAP_KINDS[self.snapshot]
        n = len(self.ops)
        self.problems = (_lib.BatchProblem * n)()
        self.bufs = []
        for slot, i in enumerate(self.order):
            op = self.ops[i]
            op.tuning = self.tuning
            plan = op._plan(dev, self.dtype)
            plan.set_tuning(*self.tuning)
            S = op.n_sources
            # the device table and the descriptors point at the plan's per-tile tables: keep these
            # tensors (and the tuning) alive even if the operator's plan is re-tuned later
            b = {"plan": plan, "S": S, "tune": plan.tuning,
                 "tables": [plan.rec_corner, plan.tile_rec_ptr, plan.tile_rec_list, plan.tile_cell_ptr,
                            plan.tile_cell_local, plan.tile_cell_gid, plan.layer_cell_index, plan.layer_cell_gid]}
            b["ring"] = plan.empty_levels(3, S)
            n_snap = -(-op.n_steps // K) if op.n_steps > 0 else 1
            b["snap"] = torch.empty(plan.snapshot_bytes(S, n_snap, kind), dtype=torch.uint8, device=dev)
            b["segbuf"] = plan.empty_levels(K, S)
            # the adjoint's q levels, and with a PML its four face-cotangent levels
            b["work"] = plan.empty_levels(7 if plan.pml is not None else 3, S, zero=False)
            if plan.pml is not None:  # the forward's face fields (the forward zeroes them)
                b["psi"] = plan.empty_levels(4, S, zero=False)
            b["acc"] = torch.empty(plan.n_acc(S), plan.field, device=dev, dtype=self.dtype)
            b["traces"] = torch.empty(S, plan.n_rec, op.n_t, device=dev, dtype=self.dtype)
            b["gtr"] = torch.zeros_like(b["traces"])
            b["c"] = torch.empty(op.domain.shape, device=dev, dtype=self.dtype)
            b["obs"] = torch.empty_like(b["traces"])
            b["c2dt2"] = torch.zeros(plan.field, device=dev, dtype=self.dtype)
            b["grad"] = torch.empty(op.domain.shape, device=dev, dtype=torch.float64)
            mask = self.masks[i]
            b["mask"] = None if mask is None else torch.as_tensor(mask).to(dev, self.dtype)
            b["loss"] = torch.empty((), device=dev, dtype=torch.float64)
            b["medium"] = plan.medium(b["c2dt2"])
            b["acq"] = plan.acquisition(S)
            st = _lib.Storage()
            st.ring, st.snap, st.segbuf = b["ring"].data_ptr(), b["snap"].data_ptr(), b["segbuf"].data_ptr()
            st.segment, st.snap_kind = K, kind
            if plan.pml is not None:
                st.pml_psi = b["psi"].data_ptr()
            q = self.problems[slot]
            q.grid, q.medium, q.acq, q.time, q.storage = plan.g, b["medium"], b["acq"], plan.time, st
            q.work, q.grad_acc = b["work"].data_ptr(), b["acc"].data_ptr()
            q.traces, q.grad_traces = b["traces"].data_ptr(), b["gtr"].data_ptr()
            self.bufs.append(b)
        self.tune = self.bufs[0]["tune"]
        self.table = torch.empty(int(lib.nw_batch_table_bytes(n)), dtype=torch.uint8, device=dev)
        _lib.check(lib.nw_batch_prepare(self.problems, n, C.byref(self.tune), self.table.data_ptr(),
                                        _lib.stream_handle(dev)))

    def memory_bytes(self) -> int:
        """Device bytes the batch holds (wavefield storage, snapshots, traces, accumulators)."""
        return sum(t.numel() * t.element_size() for b in self.bufs for t in b.values()
                   if isinstance(t, torch.Tensor)) + self.table.numel()

    # -- one gradient ---------------------------------------------------------------------------
    @_lib.on_device
    def _step(self) -> None:
        """The whole batched gradient from the static inputs (``c``, ``obs``) to the outputs."""
        lib = _lib.load()
        s = _lib.stream_handle(self.device)
        n = len(self.ops)
        for slot, i in enumerate(self.order):
            b, op = self.bufs[slot], self.ops[i]
            _lib.check(lib.nw_prepare_medium(C.byref(b["plan"].g), b["plan"].n_abs, b["c"].data_ptr(),
                                             op.dt**2, b["c2dt2"].data_ptr(), s))
        _lib.check(lib.nw_batch_forward(self.problems, n, C.byref(self.tune), self.table.data_ptr(), s))
        if self.misfits is None:
            for b in self.bufs:
                torch.sub(b["traces"], b["obs"], out=b["gtr"])
                b["loss"].copy_(0.5 * b["gtr"].double().square().sum())
        else:  # the fused pass: observation terms, then loss and adjoint source straight into gtr
            for slot, i in enumerate(self.order):
                b, mf = self.bufs[slot], self.misfits[i]
                mf.prepare(b["obs"], b["mask"], always=True)
                loss, _ = mf.value_and_grad(b["traces"], out=b["gtr"])
                b["loss"].copy_(loss)
        _lib.check(lib.nw_batch_adjoint(self.problems, n, C.byref(self.tune), self.table.data_ptr(), s))
        for slot, i in enumerate(self.order):
            b, op = self.bufs[slot], self.ops[i]
            _lib.check(lib.nw_reduce_grad_c(C.byref(b["plan"].g), b["plan"].n_abs, b["c"].data_ptr(), op.dt**2,
                                            b["acc"].shape[0], b["acc"].data_ptr(), 0, b["grad"].data_ptr(), s))

    def _load(self, cs, observed) -> None:
        if len(cs) != len(self.ops) or len(observed) != len(self.ops):
            raise ConfigError(f"expected {len(self.ops)} models and observed trace sets")
        for slot, i in enumerate(self.order):
            op = self.ops[i]
            c = cs[i]
            op._validate(c.to(self.device))
            self.bufs[slot]["c"].copy_(c, non_blocking=True)
            self.bufs[slot]["obs"].copy_(observed[i], non_blocking=True)

    def _outputs(self):
        losses = [None] * len(self.ops)
        grads = [None] * len(self.ops)
        for slot, i in enumerate(self.order):
            losses[i] = self.bufs[slot]["loss"]
            grads[i] = self.bufs[slot]["grad"]
        return losses, grads

    @_lib.on_device
    def misfit_gradients(self, cs: Sequence[torch.Tensor], observed: Sequence[torch.Tensor]):
        """``(losses, grads)``: per problem, in the order the operators were given; the gradients are
        float64 (the tensors are reused by the next call: clone to keep them)."""
        self._load(cs, observed)
        if self._graph is not None:
            self._graph.replay()
        else:
            self._step()
            self.check_snapshots()
        return self._outputs()

    @_lib.on_device
    def check_snapshots(self) -> None:
        """Synchronise and raise if a 16-bit snapshot block held a non-finite value."""
        if self.snapshot == "exact":
            return
        rc = _lib.load().nw_status(_lib.stream_handle(self.device))
        if rc == _lib.NW_ERR_NONFINITE:
            from ._compat import SolverError
            raise SolverError("a wavefield snapshot held a non-finite value: a forward run diverged")
        _lib.check(rc)

    @_lib.on_device
    def capture(self) -> None:
        """Record the whole gradient as one CUDA graph; later ``misfit_gradients`` calls replay it.
        Runs the gradient once first (on the current inputs) so that every kernel's shared-memory
        opt-in happens outside the capture."""
        torch.cuda.synchronize(self.device)
        self._step()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        lib = _lib.load()
        n0 = lib.nw_launch_count()
        with torch.cuda.graph(g):
            self._step()
        self.graph_launches = int(lib.nw_launch_count() - n0)  # this library's kernels per replay
        self._graph = g
        torch.cuda.synchronize(self.device)


@_lib.on_device
def autotune(ops: Sequence[WaveOperatorB200], *, steps: int = 120, device="cuda", dtype=torch.float32,
             snapshot: str = "delta16", fwd_candidates=((4, 2, 2), (2, 4, 2), (4, 2, 1), (2, 2, 2), (4, 4, 1)),
             adj_candidates=((2, 2, 4), (2, 2, 2), (4, 2, 4), (2, 4, 4), (2, 2, 8)), repeats: int = 2):
    """Choose the forward and adjoint tile shapes ``(vz, rx, shots_per_cta)`` for a batch by timing
    each candidate's sweep on the device over a copy of the batch shortened in time: the longest
    problem to ``steps`` samples and every other one in proportion, so that the shortened batch runs
    the same mix of problems over its steps as the real one (the per-step cost of a problem does
    not depend on the step count). Returns the 6-tuple tuning and the timings (seconds)."""
    short = []
    n_t_max = max(op.n_t for op in ops)
    for op in ops:
        n_t = max(2, min(op.n_t, round(op.n_t * (steps + 1) / n_t_max)))
        short.append(WaveOperatorB200(op.domain, op.sources, op.receivers, f0=op.f0, t0=op.t0,
                                      amplitude=op.amplitude, **{**op._kwargs(), "n_t": n_t}))
    dev = torch.device(device)
    cs = [torch.full(op.domain.shape, 0.9 * op.c_max, device=dev, dtype=dtype) for op in short]
    results = {}

    def sweep_time(tuning, which):
        bt = BatchedFWI(short, device=dev, dtype=dtype, snapshot=snapshot, tuning=tuning)
        for slot, i in enumerate(bt.order):
            bt.bufs[slot]["c"].copy_(cs[i])
        lib, s = _lib.load(), _lib.stream_handle(dev)
        n = len(short)
        for slot in range(n):
            _lib.check(lib.nw_prepare_medium(C.byref(bt.bufs[slot]["plan"].g), bt.bufs[slot]["plan"].n_abs,
                                             bt.bufs[slot]["c"].data_ptr(), short[bt.order[slot]].dt**2,
                                             bt.bufs[slot]["c2dt2"].data_ptr(), s))
        if which == "adj":  # the adjoint decodes the snapshots the forward sweep writes
            _lib.check(lib.nw_batch_forward(bt.problems, n, C.byref(bt.tune), bt.table.data_ptr(), s))
        fn = lib.nw_batch_forward if which == "fwd" else lib.nw_batch_adjoint
        best = float("inf")
        for r in range(repeats + 1):  # the device time of the sweep, the first run untimed
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.check(fn(bt.problems, n, C.byref(bt.tune), bt.table.data_ptr(), s))
            e1.record()
            torch.cuda.synchronize(dev)
            if r:
                best = min(best, e0.elapsed_time(e1) * 1e-3)
        bt.check_snapshots()
        del bt
        return best

    best_f = min(fwd_candidates, key=lambda t: results.setdefault(("fwd", t), sweep_time((*t, 0, 0, 0), "fwd")))
    best_a = min(adj_candidates,
                 key=lambda t: results.setdefault(("adj", t), sweep_time((*best_f, *t), "adj")))
    return (*best_f, *best_a), results
