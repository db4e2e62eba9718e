"""The allocation-free gradient entry point, called through the C ABI.

Some callers cannot allocate device memory: a service that reaches the propagator only through the C
ABI and owns no CUDA allocator, one that reserves its memory at start-up, or a loop that must not
call cudaMalloc because it synchronises the device. `nw_adjoint_grad_c_noalloc` serves them by taking
its adjoint scratch from a fixed array inside the library. These tests check that it returns the
gradient of the allocating path (`nw_adjoint` + `nw_reduce_grad_c`) on two calls in a row, which also
shows that the array's leftover contents from the first call do not leak into the second, and that
requests larger than the array are refused with a clear error before any GPU work.

This file sorts last so that a run stopping at the first failure has run every other test first.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import cotangent, load_golden, rel_l2
from nefi_b200 import WaveOperatorB200, _lib
from nefi_b200._compat import Domain
from nefi_b200.operators import _adjoint_sweep, _forward_sweep, _Run

pytestmark = pytest.mark.gpu

# the gradient tolerances the parity tests use (relative L2)
TOL = {torch.float64: 1e-10, torch.float32: 1e-4}


def _fwi3d_case() -> dict:
    """A small 3-D FWI geometry (sponge, order 2): the 3-D adjoint keeps one accumulator per shot."""
    return {"shape": (14, 12, 10), "extent": ((0.0, 1.4), (0.0, 1.2), (0.0, 1.0)),
            "sources": np.array([[0.5, 0.4, 0.25], [0.9, 0.7, 0.35]]),
            "receivers": np.array([[0.3 + 0.2 * i, 0.6, 0.15] for i in range(4)]),
            "c": 2.0 + 0.2 * np.random.default_rng(4).random((14, 12, 10)), "seed": 11,
            "kw": dict(n_t=30, dt_obs=0.012, f0=5.0, c_max=2.4, order=2, absorbing="sponge",
                       absorb_width=0.2)}


# (case, storage mode, snapshot kind): each lays out the shared array differently -- the sponge's three
# adjoint levels and one accumulator per shot group, the PML's seven levels (face cotangents) and one
# accumulator per shot, the 3-D adjoint's accumulator per shot, and checkpointed runs that decode
# snapshots and recompute each segment into the caller's segment buffer
CASES = [("fwi_o4_sponge", ("history", None), "exact"),
         ("fwi_o4_pml", ("history", None), "exact"),
         ("fwi3d", ("history", None), "exact"),
         ("fwi_o4_sponge", ("checkpoint", 7), "delta16"),
         ("fwi_o4_pml", ("checkpoint", 6), "exact")]


def _setup(case, dtype, dev, mode=("history", None), snapshot="exact"):
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    op = WaveOperatorB200(dom, case["sources"], case["receivers"], grad_mode="autograd", **case["kw"])
    plan = op._plan(dev, dtype)
    lib = _lib.load()
    stream = _lib.stream_handle(dev)
    c = torch.tensor(case["c"], dtype=dtype, device=dev)
    c2dt2 = torch.empty(plan.field, dtype=dtype, device=dev)
    _lib.check(lib.nw_prepare_medium(C.byref(plan.g), plan.n_abs, c.data_ptr(), op.dt**2, c2dt2.data_ptr(),
                                     stream))
    medium = plan.medium(c2dt2)
    S = op.n_sources
    acq = plan.acquisition(S)
    run = _Run(plan, S, op.n_steps, mode, snapshot)
    traces = torch.empty(S, plan.n_rec, op.n_t, dtype=dtype, device=dev)
    _forward_sweep(plan, medium, acq, run, 0, op.n_steps, traces, stream)
    g = torch.tensor(cotangent(traces.shape, case["seed"]), dtype=dtype, device=dev)
    # the descriptors hold raw device pointers: keep the tensors behind them alive
    return op, plan, lib, stream, c, medium, acq, run, g, c2dt2


@pytest.mark.parametrize("name,mode,snapshot", CASES)
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_gradient_matches_allocating_path_twice(name, mode, snapshot, dtype, cuda_device):
    case = _fwi3d_case() if name == "fwi3d" else load_golden(name)
    op, plan, lib, stream, c, medium, acq, run, g, _c2dt2 = _setup(case, dtype, cuda_device, mode, snapshot)
    # the allocating path
    gC, _, _ = _adjoint_sweep(plan, medium, acq, run, g, False, stream)
    ref = torch.empty(c.shape, dtype=torch.float64, device=cuda_device)
    _lib.check(lib.nw_reduce_grad_c(C.byref(plan.g), plan.n_abs, c.data_ptr(), op.dt**2, gC.shape[0],
                                    gC.data_ptr(), 0, ref.data_ptr(), stream))
    ref_h = ref.cpu().numpy()
    for _ in range(2):
        out = torch.full(c.shape, float("nan"), dtype=torch.float64, device=cuda_device)
        _lib.check(lib.nw_adjoint_grad_c_noalloc(
            C.byref(plan.g), plan.n_abs, C.byref(medium), C.byref(acq), C.byref(plan.time),
            C.byref(run.storage), C.byref(plan.tuning), c.data_ptr(), op.dt**2, g.data_ptr(),
            out.data_ptr(), stream))
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_l2(got, ref_h) < TOL[dtype]
        if "grad_c_f64" in case and snapshot == "exact":
            # and it is the reference's gradient, to the parity tolerance of this dtype
            golden = case["grad_c_f64"] if dtype == torch.float64 else case["grad_c_f32"]
            assert rel_l2(got, golden) < TOL[dtype]


def test_noalloc_refuses_requests_above_its_array(cuda_device):
    """20 float32 shots of a 552^2 padded grid need about 80 MB of scratch, above the 64 MiB array."""
    n, h = 512, 10.0
    dom = Domain((n, n), ((0.0, n * h), (0.0, n * h)))
    src = [[(k + 0.5) * n * h / 20, 1.5 * h] for k in range(20)]
    rec = [[(i + 0.5) * h, 2.5 * h] for i in range(0, n, 8)]
    op = WaveOperatorB200(dom, src, rec, n_t=3, dt_obs=1e-3, f0=10.0, c_max=4500.0, order=4,
                          absorbing="sponge", absorb_width=20 * h, courant=1.0)
    plan = op._plan(cuda_device, torch.float32)
    lib = _lib.load()
    c = torch.full((n, n), 3000.0, device=cuda_device)
    c2dt2 = torch.zeros(plan.field, device=cuda_device)
    medium = plan.medium(c2dt2)
    acq = plan.acquisition(20)
    store = _lib.Storage()
    store.history = c.data_ptr()  # never reached: the size check comes first
    out = torch.empty(c.shape, dtype=torch.float64, device=cuda_device)
    g = torch.zeros(20, plan.n_rec, op.n_t, device=cuda_device)
    rc = lib.nw_adjoint_grad_c_noalloc(C.byref(plan.g), plan.n_abs, C.byref(medium), C.byref(acq),
                                       C.byref(plan.time), C.byref(store), C.byref(plan.tuning),
                                       c.data_ptr(), op.dt**2, g.data_ptr(), out.data_ptr(),
                                       _lib.stream_handle(cuda_device))
    assert rc == _lib.NW_ERR_ARG
    msg = lib.nw_last_error().decode()
    assert "bytes of scratch" in msg and str(64 * 1024 * 1024) in msg
