#!/usr/bin/env python
"""Benchmark: FWI shot-gradients/s of the B200 acoustic propagator (forward + exact adjoint).

One step = one full FWI gradient of the 512^2 workload: 16 Ricker shots (10 Hz) over a seeded
layered model, 4000 leapfrog steps, order-4 stencil, 20-cell sponge, full wavefield history in HBM,
misfit 1/2 ||F(c) - d||^2 with its gradient w.r.t. c reduced over shots in float64.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Rank 0 prints one JSON line. Under torchrun every rank runs its own 16 shots (weak scaling) and the
float64 gradient and the scalar misfit are summed with NCCL all-reduces each step. ``--impl reference`` times the CPU
restatement of the reference algorithm (the oracle, float32, all host threads) on a bounded sample.

Other workloads (``--workload``), each printing one line of the same form:

* ``fwi_batch``: 64 uneven 2-D problems in one batched, checkpointed, graph-replayed gradient, with
  the plain path timed beside it one problem at a time and one shot at a time (whole problems over
  the ranks under torchrun);
* ``fwi_2048``: the 2048^2 workload (32 shots, 8000 steps), with ``--grad-mode checkpoint
  --snapshot delta16`` for its 16-bit checkpointed gradient;
* ``pat_256``: the 3-D photoacoustic gradient (256^3, 4 instances, 2000 steps, p0 and c);
* ``datagen_512x2``: float64 data generation from a 2x-refined ground truth;
* ``misfit_2048``: the fused band-limited misfit and adjoint source at the 2048^2 trace shape.

``--absorbing pml`` switches the 2-D workloads to the reference's default layer; ``--tuning`` sets the
launch shapes (``vz,rx,shots_per_cta,adj_vz,adj_rx,adj_shots_per_cta[,depth]``). The default line also
carries the batch (``batched``) and the checkpointed 2048^2 gradient (``checkpointed_2048``), measured
in the same run on one GPU.
"""

from __future__ import annotations

import argparse
import datetime
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
# an installed copy of the NEFI package (the offline install under baseline/_ref), when present: the
# B200 operators then subclass its Operator, and the reference arm also times its own torch operator
_REF = ROOT / "baseline" / "_ref"
if (_REF / "nefi" / "__init__.py").exists() and str(_REF) not in sys.path:
    sys.path.append(str(_REF))
METRIC = "FWI shot-gradients/s & Gcell-updates/s at 1e-4 grad err vs FP64; plain vs batched"
UNIT = "shot-gradients/s"
CPU_SAMPLE_SHOTS, CPU_SAMPLE_STEPS = 8, 300
REF_SAMPLE_STEPS = 100  # per reference-arm step: every shot of the workload for this many steps


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_desc(w, storage: str = "full history in HBM", layer: str = "sponge") -> dict:
    P = w.n + 2 * w.absorb_cells
    model = ("seeded layered model (6-10 layers 1500-4500 m/s + 4 anomalies) + salt body (4500 m/s)"
             if w.name == "fwi_2048" else "seeded layered model (6-10 layers 1500-4500 m/s + 4 anomalies)")
    return {"workload": f"{w.name}: {w.n}x{w.n} FP32 grid h={w.h:g} m, {model}, {len(w.sources)} Ricker shots "
                        f"{w.f0:g} Hz, {len(w.receivers)} receivers, {w.n_steps} steps, Courant "
                        f"{w.courant_number}, order {w.order}, {w.absorb_cells}-cell {layer}, {storage}",
            "grid_padded": [P, P], "shots_per_gpu": len(w.sources), "n_steps": w.n_steps,
            "l2": "256 MiB buffer written between timed steps; working set (history) far above L2"}


# ------------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.count(",") >= 8]
        self.path.unlink(missing_ok=True)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].strip().replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].strip().replace(".", "").isdigit())}


# ------------------------------------------------------------------------------------------------
# CPU baseline: the oracle (float32, all host threads) on a bounded sample of the workload
# ------------------------------------------------------------------------------------------------
def cpu_sample(w, n_shots=CPU_SAMPLE_SHOTS, n_steps=CPU_SAMPLE_STEPS) -> tuple[float, dict]:
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # noqa: E402  (the checker, used here only as the timed CPU baseline)

    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    n_steps = max(20, min(n_steps, int(n_steps * 552**2 / (w.n + 2 * w.absorb_cells) ** 2)))  # ~10-30 s of CPU
    kw = w.operator_kwargs()
    kw["n_t"] = n_steps + 1
    L = w.n * w.h
    orc = oracle.OracleWave((w.n, w.n), ((0.0, L), (0.0, L)), w.receivers, sources=w.sources[:n_shots],
                            **{k: v for k, v in kw.items()})
    g = np.random.default_rng(1).standard_normal((n_shots, len(w.receivers), n_steps + 1)).astype(np.float32)
    t0 = time.perf_counter()
    orc.fwi(w.c, g, dtype=np.float32)
    t = time.perf_counter() - t0
    per_shot_full = t / n_shots * (w.n_steps / n_steps)
    info = {"cores": min(threads, n_shots), "sample": f"{n_shots} shots x {n_steps} of {w.n_steps} steps "
            f"(forward + adjoint, full {w.n + 2 * w.absorb_cells}^2 padded grid), float32; measured {t:.2f} s, "
            f"extrapolated linearly in steps", "seconds": t, "steps": n_steps,
            "gcell_updates_per_s": 2 * w.padded_cells() * n_steps * n_shots / t / 1e9}
    return 1.0 / per_shot_full, info


def make_workload(args):
    from nefi_b200 import workloads

    kw = {}
    if getattr(args, "n_steps", None):
        kw["n_steps"] = args.n_steps
    if getattr(args, "shots", None):
        kw["n_shots"] = args.shots
    return workloads.WORKLOADS[args.workload](**kw)


def measure_batch(dev, world: int, rank: int, n_problems: int = 64, steps: int = 3, warmup: int = 3,
                  snapshot: str = "delta16", n_steps: int | None = None, with_plain: bool = True,
                  with_e2e: bool = True, accuracy_problems: int = 0) -> dict:
    """The uneven batch (seeded 2-D problems, 256-768^2, 4-16 shots, 1500-6000 steps) in one batched,
    checkpointed (16-bit snapshots), graph-replayed gradient; with the plain one-problem-at-a-time
    path timed beside it, the end-to-end figure, and the float32 gradient error against float64 runs
    of ``accuracy_problems`` of the problems. Returns the bench line's fields."""
    import torch.distributed as dist

    from nefi_b200 import WaveOperatorB200, workloads
    from nefi_b200.batched import BatchedFWI, autotune
    from nefi_b200.distributed import problem_shards

    ws_all = workloads.fwi_batch_problems(seed=0, n_problems=n_problems)
    if n_steps:  # shortened case for profiling: steps scaled to at most n_steps
        for w in ws_all:
            w.n_steps = max(2, round(w.n_steps * n_steps / 6000))
    # whole problems over the ranks, balanced by shots x cells x steps (no collective on the data path)
    mine = problem_shards([len(w.sources) * w.padded_cells() * w.n_steps for w in ws_all], world)[rank]
    ws = [ws_all[i] for i in mine]

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t)
    single_shot = None
    if with_plain:
        # the plain single-shot path, measured before the batch allocates its storage: one shot per
        # operator call (the full history in HBM where it fits), on one shot of the first problem of
        # each grid size, scaled to the whole batch by useful cell-updates
        firsts = {}
        for i, w in enumerate(ws):
            firsts.setdefault(w.n, i)
        single = []
        for i in firsts.values():
            w = ws[i]
            k = len(w.sources) // 2
            op1 = WaveOperatorB200(w.domain, [w.sources[k]], w.receivers, grad_mode="autograd",
                                   **w.operator_kwargs())
            c1 = torch.tensor(w.c, dtype=torch.float32, device=dev)
            with torch.no_grad():
                d1 = op1({"c": torch.nn.functional.avg_pool2d(c1[None, None], 9, 1, 4, count_include_pad=False)[0, 0]
                                .contiguous()})
            op1.misfit_gradient(c1, d1)  # plan, allocation, kernel loading
            single.append((op1, c1, d1, 2 * w.padded_cells() * w.n_steps,
                           f"{w.n}^2 x {w.n_steps} steps, 1 shot, {op1.last_storage[0] if op1.last_storage else '?'}"))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for op1, c1, d1, _, _ in single:
            op1.misfit_gradient(c1, d1)
        e1.record()
        torch.cuda.synchronize()
        single_ms = max_over_ranks(e0.elapsed_time(e1))
        rate = sum(s[3] for s in single) / (single_ms * 1e-3)  # useful cell-updates/s, one shot per call
        useful_all = sum(2 * w.padded_cells() * w.n_steps * len(w.sources) for w in ws_all)
        single_shot = {
            "value": sum(len(w.sources) for w in ws_all) / (useful_all / rate), "unit": UNIT,
            "gcell_updates_per_s": rate / 1e9, "measured_ms": single_ms, "sample": [s[4] for s in single],
            "method": "one shot per WaveOperatorB200.misfit_gradient call, grad_mode='autograd' (the full "
                      "history in HBM where it fits), measured before the batch allocates; the sample's "
                      "useful cell-updates/s applied to the whole batch's useful cell-updates"}
        del single, op1
        torch.cuda.empty_cache()
    ops = [WaveOperatorB200(w.domain, w.sources, w.receivers, grad_mode="checkpoint", snapshot=snapshot,
                            **w.operator_kwargs()) for w in ws]
    cs = [torch.tensor(w.c, dtype=torch.float32, device=dev) for w in ws]
    with torch.no_grad():
        obs = [op({"c": torch.nn.functional.avg_pool2d(c[None, None], 9, 1, 4, count_include_pad=False)[0, 0]
                         .contiguous()}) for op, c in zip(ops, cs)]
    t0 = time.perf_counter()
    tuning, _ = autotune(ops, steps=200, device=dev, repeats=2, snapshot=snapshot)
    t_tune = time.perf_counter() - t0
    bt = BatchedFWI(ops, device=dev, snapshot=snapshot, tuning=tuning)
    bt.misfit_gradients(cs, obs)
    t0 = time.perf_counter()
    bt.capture()
    t_capture = time.perf_counter() - t0
    flush = torch.empty(64 * 2**20, dtype=torch.float32, device=dev)
    for _ in range(warmup):
        bt.misfit_gradients(cs, obs)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(dev.index)
    times = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        bt._graph.replay()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    bt.check_snapshots()
    ms = max_over_ranks(sum(times) / len(times))
    shots = sum(len(w.sources) for w in ws_all)
    useful = sum(2 * w.padded_cells() * w.n_steps * len(w.sources) for w in ws_all)
    recompute = sum(w.padded_cells() * w.n_steps * len(w.sources) for w in ws_all)
    peak, peak_kind = peaks()
    achieved = 16.0 * useful / (ms * 1e-3) / 1e9
    accuracy = None
    if accuracy_problems > 0:
        # the batch's float32 gradients (16-bit snapshots) against float64 runs of the same problems
        # alone (exact checkpoints), for the problems with the least work
        _, grads = bt._outputs()
        pick = sorted(range(len(ws)), key=lambda i: len(ws[i].sources) * ws[i].padded_cells() * ws[i].n_steps)
        errs, fixed = {}, {}
        for i in pick[:accuracy_problems]:
            g32 = grads[i].clone()
            w = ws[i]
            name = f"problem{mine[i]} ({w.n}^2, {len(w.sources)} shots, {w.n_steps} steps)"
            op64 = WaveOperatorB200(w.domain, w.sources, w.receivers, grad_mode="checkpoint", **w.operator_kwargs())
            _, g64 = op64.misfit_gradient(cs[i].double(), obs[i].double())
            errs[name] = float((g32 - g64).norm() / g64.norm())
            fixed[name] = fixed_cotangent_error(op64, WaveOperatorB200(
                w.domain, w.sources, w.receivers, grad_mode="checkpoint", snapshot=snapshot, checkpoint_every=bt.segment,
                **w.operator_kwargs()), cs[i], obs[i])
            del op64, g64
        accuracy = {"grad_rel_l2_fp32_vs_fp64": max(errs.values()), "per_problem": errs,
                    "fixed_cotangent": {"grad_rel_l2_fp32_vs_fp64": max(v["grad"] for v in fixed.values()),
                                        "per_problem": fixed},
                    "fp32_storage": f"checkpointed, {snapshot} snapshots, segment {bt.segment}",
                    "fp64_storage": "checkpointed, exact snapshots",
                    "note": "grad_rel_l2_fp32_vs_fp64: each precision's own misfit gradient (its own residual); "
                            "fixed_cotangent: the float32 adjoint given the float64 residual, which isolates the "
                            "adjoint and the snapshots from the float32 rounding of the traces that the residual "
                            "magnifies by ||traces|| / ||residual|| (resid_ratio)"}
    out = {"value": shots / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": warmup,
           "config": {"workload": f"fwi_batch: {len(ws_all)} problems, grids {{256,384,512,768}}^2 + 20-cell sponge, "
                                  f"4-16 Ricker shots, 1500-6000 steps (seed 0), order 4; checkpointed with "
                                  f"{snapshot} snapshots, segment {bt.segment}; one launch per step over all running "
                                  f"problems, whole gradient replayed from one CUDA graph",
                      "method": "batched", "shots_total": shots, "tuning": list(tuning),
                      "parallelism": f"whole problems balanced by cost over {world} GPU(s); no collective",
                      "autotune_s": t_tune, "graph_capture_s": t_capture,
                      "device_bytes": bt.memory_bytes(),
                      "l2": "256 MiB buffer written between timed steps; working set far above L2"},
           "gcell_updates_per_s": useful / (ms * 1e-3) / 1e9,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": None, "peak_source": peak_kind,
                        "note": "16 B per useful cell-update (forward + adjoint) over the CUDA-event time of the "
                                f"replays; the segment recompute ({recompute / 1e9:.0f} G extra cell-updates per "
                                "gradient) is not counted",
                        "kernel_rate_GBps_incl_recompute": 16.0 * (useful + recompute) / (ms * 1e-3) / 1e9},
           "accuracy": accuracy, "clocks": clocks, "gpu_launches": bt.graph_launches * steps}
    if with_plain:
        # the plain path on the same problems, one problem at a time (same storage, default tuning)
        for op in ops:
            op.tuning = None
            op._plans.clear()
        ops[0].misfit_gradient(cs[0], obs[0])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for op, c, d in zip(ops, cs, obs):
            op.misfit_gradient(c, d)
        e1.record()
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(e0.elapsed_time(e1))
        out["plain"] = {"value": shots / (plain_ms * 1e-3), "unit": UNIT, "ms_per_gradient_of_all_problems": plain_ms,
                        "method": "each problem alone through WaveOperatorB200.misfit_gradient (same storage)"}
        out["plain_single_shot"] = single_shot

    if with_e2e:
        # end to end: models and observed data from pinned host memory in, gradients and losses out
        c_h = [c.cpu().pin_memory() for c in cs]
        d_h = [d.cpu().pin_memory() for d in obs]
        g_h = [torch.empty(c.shape, dtype=torch.float64).pin_memory() for c in cs]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        losses, grads = bt.misfit_gradients([c.to(dev, non_blocking=True) for c in c_h],
                                            [d.to(dev, non_blocking=True) for d in d_h])
        for g, gh in zip(grads, g_h):
            gh.copy_(g, non_blocking=True)
        loss_h = torch.stack(losses).cpu()
        e1.record()
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1))
        h2d = sum(t.numel() * t.element_size() for t in c_h + d_h)
        d2h = sum(t.numel() * 8 for t in g_h) + loss_h.numel() * 8
        if world > 1:  # whole-job bytes per step
            t = torch.tensor([float(h2d), float(d2h)], dtype=torch.float64, device=dev)
            dist.all_reduce(t)
            h2d, d2h = int(t[0]), int(t[1])
        out["e2e"] = {"value": shots / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                      "d2h_bytes_per_step": d2h}
    bt._graph = None
    del bt
    torch.cuda.empty_cache()
    return out


def fixed_cotangent_error(op64, op32, c, obs) -> dict:
    """The float32 gradient of ``op32`` given the float64 residual of ``op64`` as the trace cotangent,
    against the float64 gradient: the error of the adjoint sweep and its storage alone. Also the
    float32 traces' error and the residual's size relative to the traces."""
    c64 = c.double().clone().requires_grad_(True)
    tr64 = op64({"c": c64})
    r64 = (tr64 - obs.double()).detach()
    (g64,) = torch.autograd.grad((tr64 * r64).sum(), c64)
    c32 = c.float().clone().requires_grad_(True)
    tr32 = op32({"c": c32})
    (g32,) = torch.autograd.grad((tr32 * r64.float()).sum(), c32)
    out = {"grad": float((g32.double() - g64).norm() / g64.norm()),
           "traces": float((tr32.detach().double() - tr64.detach()).norm() / tr64.detach().norm()),
           "resid_ratio": float(tr64.detach().norm() / r64.norm())}
    del c64, tr64, r64, g64, c32, tr32, g32
    torch.cuda.empty_cache()
    return out


def measure_checkpointed(dev, w, snapshot: str = "delta16", steps: int = 1, warmup: int = 1,
                         accuracy_shots: int = 4) -> dict:
    """One FWI gradient of workload ``w`` with checkpointed storage and 16-bit snapshots (the large
    configuration's method), CUDA-event timed; with the float32 gradient error against a float64 run
    (exact snapshots) over the first ``accuracy_shots`` shots. Returns the bench line's fields."""
    from nefi_b200 import WaveOperatorB200
    from nefi_b200.plan import plan_storage

    op = WaveOperatorB200(w.domain, w.sources, w.receivers, grad_mode="checkpoint", snapshot=snapshot,
                          **w.operator_kwargs())
    c = torch.tensor(w.c, dtype=torch.float32, device=dev)
    with torch.no_grad():
        d = op({"c": torch.nn.functional.avg_pool2d(c[None, None], 9, 1, 4, count_include_pad=False)[0, 0]
                .contiguous()})
    mode = plan_storage(op._plan(dev, torch.float32), len(w.sources), op.n_steps, op.grad_mode,
                        op.checkpoint_every, op.snapshot, op._budget(dev))
    flush = torch.empty(64 * 2**20, dtype=torch.float32, device=dev)
    for _ in range(warmup):
        op.misfit_gradient(c, d)
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index)
    times = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        op.misfit_gradient(c, d)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    ms = sum(times) / len(times)
    S = len(w.sources)
    useful = 2 * w.padded_cells() * w.n_steps * S
    peak, peak_kind = peaks()
    achieved = 16.0 * useful / (ms * 1e-3) / 1e9
    accuracy = None
    if accuracy_shots > 0:
        na = accuracy_shots
        op32 = WaveOperatorB200(w.domain, w.sources[:na], w.receivers, grad_mode="checkpoint", snapshot=snapshot,
                                **w.operator_kwargs())
        _, g32 = op32.misfit_gradient(c, d[:na])
        del op32
        op64 = WaveOperatorB200(w.domain, w.sources[:na], w.receivers, grad_mode="checkpoint", **w.operator_kwargs())
        _, g64 = op64.misfit_gradient(c.double(), d[:na].double())
        fixed = fixed_cotangent_error(op64, WaveOperatorB200(
            w.domain, w.sources[:na], w.receivers, grad_mode="checkpoint", snapshot=snapshot,
            checkpoint_every=mode[1], **w.operator_kwargs()), c, d[:na])
        accuracy = {"grad_rel_l2_fp32_vs_fp64": float((g32 - g64).norm() / g64.norm()), "shots": na,
                    "fixed_cotangent": fixed,
                    "fp32_storage": f"checkpointed every {mode[1]} steps, {snapshot} snapshots",
                    "fp64_storage": "checkpointed, exact snapshots"}
        del op64, g32, g64
    del op, c, d
    torch.cuda.empty_cache()
    return {"value": S / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": warmup,
            "config": workload_desc(w, f"checkpointed every {mode[1]} steps with {snapshot} snapshots"),
            "gcell_updates_per_s": useful / (ms * 1e-3) / 1e9,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                         "note": "16 B per useful cell-update (forward + adjoint) over the CUDA-event time of "
                                 "the whole gradient; the segment recompute is not counted"},
            "accuracy": accuracy, "clocks": clocks}


def run_batch(args) -> None:
    """``--workload fwi_batch``: the batch's own bench line (whole problems over the ranks under
    torchrun, no collective on the data path)."""
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    snapshot = args.snapshot if args.snapshot != "exact" else "delta16"
    m = measure_batch(dev, world, rank, args.problems, args.steps, args.warmup, snapshot, args.n_steps,
                      accuracy_problems=0 if args.no_accuracy else 4)
    out = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (64 seeded layered models; observed data from smoothed models)",
           **{k: v for k, v in m.items() if k not in ("value", "unit", "ms_per_step", "steps", "warmup")}}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_pat(args) -> None:
    """3-D photoacoustic gradient: 256^3 grid + 20-cell sponge, c = 1500 m/s
    +-5 % smooth seeded perturbation, 4 instances of 20 random ellipsoids, a 256 x 256 sensor plane,
    2000 steps; the gradient w.r.t. p0 and c of 1/2 ||F(p0) - d||^2, checkpointed storage."""
    from nefi_b200 import WaveInitialConditionOperatorB200, workloads

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n_steps = args.n_steps or 2000
    n = args.pat_n
    w = workloads.pat_volume(n=n, batch=4, n_steps=n_steps)
    op = WaveInitialConditionOperatorB200(w.domain, w.sensors, grad_mode="checkpoint", snapshot=args.snapshot,
                                          checkpoint_every=args.checkpoint_every, **w.operator_kwargs())
    p0 = torch.tensor(w.p0, device=dev)
    c = torch.tensor(w.c, dtype=torch.float32, device=dev)
    with torch.no_grad():
        d = op({"p0": p0 * 0.9})

    def step():
        x = p0.clone().requires_grad_(True)
        cc = c.clone().requires_grad_(True)
        tr = op.with_speed(x, cc)
        loss = 0.5 * (tr - d).double().square().sum()
        gp, gc = torch.autograd.grad(loss, (x, cc))
        return loss, gp, gc

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    lib = __import__("nefi_b200")._lib.load()
    l0 = lib.nw_launch_count()
    sampler = ClockSampler(dev.index)
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    launches = lib.nw_launch_count() - l0
    ms = sum(times) / len(times)
    P = op.grid.padded_shape
    cells = P[0] * P[1] * P[2]
    # end to end: p0, c and the observed traces from pinned host memory, both gradients and the loss back
    p0_h, c_h, d_h = p0.cpu().pin_memory(), c.cpu().pin_memory(), d.cpu().pin_memory()
    gp_h = torch.empty(p0.shape, dtype=p0.dtype).pin_memory()
    gc_h = torch.empty(c.shape, dtype=c.dtype).pin_memory()
    e2e = []
    for i in range(1 + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        x = p0_h.to(dev, non_blocking=True).requires_grad_(True)
        cc = c_h.to(dev, non_blocking=True).requires_grad_(True)
        dd = d_h.to(dev, non_blocking=True)
        loss = 0.5 * (op.with_speed(x, cc) - dd).double().square().sum()
        gp, gc = torch.autograd.grad(loss, (x, cc))
        gp_h.copy_(gp, non_blocking=True)
        gc_h.copy_(gc, non_blocking=True)
        loss.detach().cpu()
        e1.record()
        torch.cuda.synchronize()
        if i:
            e2e.append(e0.elapsed_time(e1))
        del x, cc, dd, gp, gc, loss
    e2e_ms = statistics.median(e2e)
    h2d = sum(t.numel() * t.element_size() for t in (p0_h, c_h, d_h))
    d2h = gp_h.numel() * gp_h.element_size() + gc_h.numel() * gc_h.element_size() + 8
    accuracy = None
    if not args.no_accuracy:
        # the float32 gradients of instance 0 (this run's storage and snapshots) against a float64 device
        # run of the same instance (exact checkpoints); tests/test_gpu_parity.py checks that float64
        # path against the float64 oracle on a 96^3 grid
        def grads(dtype, snapshot):
            o = WaveInitialConditionOperatorB200(w.domain, w.sensors, grad_mode="checkpoint", snapshot=snapshot,
                                                 checkpoint_every=args.checkpoint_every, **w.operator_kwargs())
            x = p0[:1].to(dtype).clone().requires_grad_(True)
            cc = c.to(dtype).clone().requires_grad_(True)
            lo = 0.5 * (o.with_speed(x, cc) - d[:1].to(dtype)).double().square().sum()
            return torch.autograd.grad(lo, (x, cc))
        gp32, gc32 = grads(torch.float32, args.snapshot)
        torch.cuda.empty_cache()
        gp64, gc64 = grads(torch.float64, "exact")
        accuracy = {"grad_p0_rel_l2_fp32_vs_fp64": float((gp32.double() - gp64).norm() / gp64.norm()),
                    "grad_c_rel_l2_fp32_vs_fp64": float((gc32.double() - gc64).norm() / gc64.norm()),
                    "instances": 1, "fp32_storage": f"checkpointed, {args.snapshot} snapshots",
                    "fp64_storage": "checkpointed, exact snapshots"}
        del gp32, gc32, gp64, gc64
        torch.cuda.empty_cache()
    cpu = None
    if not args.no_cpu_baseline:
        # the float32 C oracle (all host threads) on one instance and a few steps of the same grid,
        # forward and adjoint with the p0 and c gradients, extrapolated to the workload
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle  # noqa: E402  (the checker, used here only as the timed CPU baseline)

        oracle.set_threads(os.cpu_count() or 1)
        kw = dict(w.operator_kwargs())
        cs_ = kw.pop("c").numpy()

        def oracle_seconds(n_t):
            orc = oracle.OracleWave(w.domain.shape, w.domain.extent, w.sensors, c_max=float(cs_.max()),
                                    **{**kw, "n_t": n_t})
            g_s = np.random.default_rng(1).standard_normal((1, len(w.sensors), n_t)).astype(np.float32)
            t0 = time.perf_counter()
            orc.pat(w.p0[:1], cs_, g_s, dtype=np.float32)
            return time.perf_counter() - t0

        # the per-step cost from two sample lengths (the setup each run repeats cancels out)
        t_a, t_b = oracle_seconds(3), oracle_seconds(9)
        steps_done = 6 * op.substeps
        per_step = max(t_b - t_a, 1e-9) / steps_done
        cpu = {"value": 1.0 / (per_step * op.n_steps), "unit": "instance-gradients/s",
               "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"1 instance, runs of {2 * op.substeps} and {8 * op.substeps} of {op.n_steps} steps "
                         f"(forward + adjoint, p0 and c gradients) on the {P[0]}^3 padded grid, float32; the "
                         "difference of the two times per step, times the workload's steps",
               "gcell_updates_per_s": 2 * cells / per_step / 1e9}
    useful = 2 * cells * op.n_steps * 4
    peak, peak_kind = peaks()
    achieved = 16.0 * useful / (ms * 1e-3) / 1e9
    out = {"metric": METRIC, "value": 4 / (ms * 1e-3), "unit": "instance-gradients/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded smooth speed, 20 random ellipsoids per instance)",
           "config": {"workload": f"pat_{n}: {n}^3 grid + 20-cell sponge ({P[0]}^3 padded), order 2, 4 instances, "
                                  f"{len(w.sensors)} sensors on one face, {op.n_steps} steps; gradient w.r.t. p0 and c; "
                                  f"checkpointed with {args.snapshot} snapshots",
                      "method": "plain (per-step launches)",
                      "l2": "working set (4 x {0:.0f} MB per level) far above L2".format(cells * 16 / 1e6)},
           "gcell_updates_per_s": useful / (ms * 1e-3) / 1e9,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": None, "peak_source": peak_kind,
                        "note": "16 B per useful cell-update (forward + adjoint); the segment recompute is not counted"},
           "cpu_baseline": cpu,
           "e2e": {"value": 4 / (e2e_ms * 1e-3), "unit": "instance-gradients/s", "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h},
           "accuracy": accuracy, "clocks": clocks, "gpu_launches": int(launches)}
    print(json.dumps(out), flush=True)


def run_datagen(args) -> None:
    """FP64 data generation on the device (the DataGenerator path, nefi/bench/base.py:74-90): the
    512^2 workload's operator moved to float64 and called through ``at_resolution`` with the ground
    truth on the 2x-refined 1024^2 grid (2 substeps per sample), all shots, no gradient. One step =
    the traces of every shot. The CPU baseline is the float64 oracle on a bounded sample."""
    from nefi_b200 import WaveOperatorB200, _lib

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    args.workload = "fwi_512"
    w = make_workload(args)
    op = WaveOperatorB200(w.domain, w.sources, w.receivers, **w.operator_kwargs()).to(device=dev, dtype=torch.float64)
    fine_n = 2 * w.n
    c_fine = torch.nn.functional.interpolate(torch.tensor(w.c, dtype=torch.float64)[None, None], size=(fine_n, fine_n),
                                             mode="bilinear", align_corners=False)[0, 0]
    gen = op.at_resolution((fine_n, fine_n))
    c_dev = c_fine.to(dev)
    flush = torch.empty(64 * 2**20, dtype=torch.float32, device=dev)

    def step(cc):
        with torch.no_grad():
            return gen({"c": cc})

    for _ in range(args.warmup):
        step(c_dev)
    torch.cuda.synchronize()
    lib = _lib.load()
    l0 = lib.nw_launch_count()
    sampler = ClockSampler(dev.index)
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tr = step(c_dev)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    launches = lib.nw_launch_count() - l0
    ms = statistics.median(times)
    S = len(w.sources)
    P = gen.grid.padded_shape
    cells = P[0] * P[1]
    N = gen.n_steps
    peak, peak_kind = peaks()
    alg = 32.0 * cells * S  # float64: read p^n, p^n-1, c^2 dt^2, write p^n+1
    achieved = alg / (ms / N * 1e-3) / 1e9
    # end to end: ground truth in from pinned host memory, every trace back to pinned host memory
    c_h = c_fine.pin_memory()
    tr_h = torch.empty(tr.shape, dtype=torch.float64).pin_memory()
    e2e = []
    for i in range(1 + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = step(c_h.to(dev, non_blocking=True))
        tr_h.copy_(out, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        if i:
            e2e.append(e0.elapsed_time(e1))
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle  # noqa: E402  (the checker, used here only as the timed CPU baseline)

        oracle.set_threads(os.cpu_count() or 1)
        ns, nst = 2, 400
        kw = dict(w.operator_kwargs())
        kw["n_t"] = nst // 2 + 1
        L = w.n * w.h
        orc = oracle.OracleWave((fine_n, fine_n), ((0.0, L), (0.0, L)), w.receivers, sources=w.sources[:ns], **kw)
        t0 = time.perf_counter()
        orc.fwi(c_fine.numpy(), None, dtype=np.float64)
        t = time.perf_counter() - t0
        steps_done = (kw["n_t"] - 1) * gen.substeps
        v = 1.0 / (t / ns * N / steps_done)
        cpu = {"value": v, "unit": "shot-generations/s", "cores": min(os.cpu_count() or 1, ns), "kind": "port",
               "sample": f"{ns} shots x {steps_done} of {N} steps, float64 forward on the {P[0]}^2 padded grid; "
                         "extrapolated linearly in steps",
               "gcell_updates_per_s": cells * steps_done * ns / t / 1e9}
    out = {"metric": METRIC, "value": S / (ms * 1e-3), "unit": "shot-generations/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded layered model, bilinear 2x ground truth)",
           "config": {"workload": f"datagen_512x2: fwi_512 operator (16 shots, 512 receivers, Ricker 10 Hz) generating "
                                  f"float64 traces from a {fine_n}^2 ground truth ({P[0]}^2 padded, {N} steps, "
                                  f"{gen.substeps} substeps per sample), forward only",
                      "l2": "256 MiB buffer written between timed steps; working set far above L2"},
           "gcell_updates_per_s": cells * N * S / (ms * 1e-3) / 1e9,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": None, "kernel": "fwd2d<double>", "peak_source": peak_kind,
                        "note": "32 B per float64 cell-update; launch time = step time / steps (injection included)"},
           "cpu_baseline": cpu,
           "e2e": {"value": S / (statistics.median(e2e) * 1e-3), "unit": "shot-generations/s",
                   "h2d_bytes_per_step": c_h.numel() * 8, "d2h_bytes_per_step": tr_h.numel() * 8},
           "clocks": clocks, "gpu_launches": int(launches)}
    print(json.dumps(out), flush=True)


def run_misfit(args) -> None:
    """Fused band-limited relative misfit + adjoint source at the 2048^2 workload's trace shape
    (32 shots x 2048 receivers x 8001 samples, float32), 20 Hz low-pass with a 0.3 taper and the
    sensors' 40 Hz Gaussian response, a muted-trace mask. One step = loss and dLoss/dpred of every trace.
    Beside it, the same chain as separate torch.fft calls (the unfused formulation) on the same GPU."""
    from nefi_b200 import _lib
    from nefi_b200.misfit import TraceMisfit

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    shots, rec, n_t, dt = args.shots or 32, 2048, (args.n_steps or 8000) + 1, 1e-3
    g = torch.Generator(device=dev).manual_seed(0)
    obs = torch.randn(shots, rec, n_t, device=dev, generator=g)
    pred = obs + 0.3 * torch.randn(shots, rec, n_t, device=dev, generator=g)
    mask = (torch.rand(shots, rec, 1, device=dev, generator=g) > 0.05).float()
    mf = TraceMisfit(dt, 20.0, 0.3, True, sensor_cutoff=40.0)
    mf.prepare(obs, mask)

    def step():
        mf._state[_lib.NW_MISFIT_SUM:_lib.NW_MISFIT_LOSS + 1].zero_()
        return mf.value_and_grad(pred)

    flush = torch.empty(64 * 2**20, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    lib = _lib.load()
    l0 = lib.nw_launch_count()
    sampler = ClockSampler(dev.index)
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    launches = lib.nw_launch_count() - l0
    ms = statistics.median(times)
    n_tr = shots * rec
    alg = 12.0 * n_tr * n_t + 4.0 * n_tr  # read pred and obs, write the adjoint source; the per-trace mask
    peak, peak_kind = peaks()

    # the unfused chain with torch.fft (cuFFT), for comparison: G pred - obs, low-pass, masked mean, and
    # the backward through autograd
    def fast_len(n):
        m = n
        while True:
            r = m
            for q in (2, 3, 5):
                while r % q == 0:
                    r //= q
            if r == 1:
                return m
            m += 1

    nf = fast_len(2 * n_t)
    f = torch.fft.rfftfreq(nf, d=dt, dtype=torch.float64)
    f1 = 0.7 * 20.0
    w = torch.ones_like(f)
    roll = (f > f1) & (f < 20.0)
    w[roll] = 0.5 * (1.0 + torch.cos(math.pi * (f[roll] - f1) / (20.0 - f1)))
    w[f >= 20.0] = 0.0
    w = w.float().to(dev)
    fs = torch.fft.rfftfreq(2 * n_t, d=dt, dtype=torch.float64)
    hs = torch.exp(-0.5 * (fs / 40.0) ** 2).float().to(dev)
    m_full = mask.expand_as(obs)
    of = torch.fft.irfft(torch.fft.rfft(obs, n=nf, dim=-1) * w, n=nf, dim=-1)[..., :n_t]
    den = ((of**2 * m_full).sum() / m_full.sum()).clamp_min(1e-30)

    def chain():
        x = pred.detach().requires_grad_(True)
        y = torch.fft.irfft(torch.fft.rfft(x, n=2 * n_t, dim=-1) * hs, n=2 * n_t, dim=-1)[..., :n_t]
        r = torch.fft.irfft(torch.fft.rfft(y - obs, n=nf, dim=-1) * w, n=nf, dim=-1)[..., :n_t]
        loss = (r**2 * m_full).sum() / m_full.sum() / den
        (gx,) = torch.autograd.grad(loss, x)
        return loss, gx

    chain_ms = None
    try:
        for _ in range(2):
            chain()
        torch.cuda.synchronize()
        ct = []
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            lc, gc = chain()
            e1.record()
            torch.cuda.synchronize()
            ct.append(e0.elapsed_time(e1))
        chain_ms = statistics.median(ct)
        lf, gf = step()
        chain_err = {"loss_rel": abs(float(lf) - float(lc)) / abs(float(lc)),
                     "grad_rel_l2": float((gf - gc).norm() / gc.norm())}
        del lc, gc
    except torch.OutOfMemoryError:
        chain_err = "out of memory"
    torch.cuda.empty_cache()

    # end to end: traces in from pinned host memory, the adjoint source and the loss back
    pred_h = pred.cpu().pin_memory()
    grad_h = torch.empty_like(pred_h).pin_memory()
    loss_h = torch.empty((), dtype=torch.float64).pin_memory()
    e2e = []
    for i in range(1 + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pd = pred_h.to(dev, non_blocking=True)
        mf._state[_lib.NW_MISFIT_SUM:_lib.NW_MISFIT_LOSS + 1].zero_()
        lo, gr = mf.value_and_grad(pd)
        grad_h.copy_(gr, non_blocking=True)
        loss_h.copy_(lo, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        if i:
            e2e.append(e0.elapsed_time(e1))
        del pd, gr
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import misfit_oracle  # noqa: E402  (the checker, used here only as the timed CPU baseline)

        k = 512
        ph, oh, mh = (pred[0, :k].double().cpu().numpy(), obs[0, :k].double().cpu().numpy(),
                      mask[0, :k].double().cpu().numpy())
        t0 = time.perf_counter()
        misfit_oracle.band_limited_mse(ph, oh, dt, 20.0, 0.3, True, mh, sensor=40.0)
        tc = time.perf_counter() - t0
        cpu = {"value": k / tc, "unit": "traces/s", "cores": 1, "kind": "port",
               "sample": f"{k} of {n_tr} traces, numpy pocketfft float64 (loss and gradient)"}
    out = {"metric": METRIC, "value": n_tr / (ms * 1e-3), "unit": "traces/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded gaussian traces, 5% muted)",
           "config": {"workload": f"misfit_2048: {shots} shots x {rec} receivers x {n_t} samples, band-limited "
                                  "relative MSE (f_max 20 Hz, taper 0.3) of the 40 Hz sensor-filtered prediction, "
                                  "loss and adjoint source",
                      "l2": "inputs of 2 x {0:.1f} GB, far above L2; 256 MiB written between steps".format(
                          4.0 * n_tr * n_t / 1e9)},
           "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / (ms * 1e-3) / 1e9 / peak, "traffic": None, "kernel": "misfit_fft_kernel<float>",
                        "peak_source": peak_kind,
                        "note": "12 B per sample (read pred and obs, write the adjoint source) per launch"},
           "unfused_torch_fft_ms": chain_ms, "fused_vs_unfused": chain_err,
           "cpu_baseline": cpu,
           "e2e": {"value": n_tr / (statistics.median(e2e) * 1e-3), "unit": "traces/s",
                   "h2d_bytes_per_step": pred_h.numel() * 4, "d2h_bytes_per_step": grad_h.numel() * 4 + 8},
           "clocks": clocks, "gpu_launches": int(launches)}
    print(json.dumps(out), flush=True)


def reference_torch_sample(w, n_shots: int = 4, n_steps: int = 50) -> dict | None:
    """The reference's own operator (nefi.physics.wave.WaveOperator, torch on the host cores) on a
    bounded sample of workload ``w``: forward + autograd gradient of 1/2 ||traces||^2 w.r.t. c for
    ``n_shots`` shots x ``n_steps`` steps, extrapolated linearly in shots and steps. None when the
    nefi package is not importable (an installed copy under baseline/_ref is used when present)."""
    try:
        from nefi.domain import Domain
        from nefi.physics.wave import WaveOperator
    except Exception:
        return None
    torch.set_num_threads(os.cpu_count() or 1)
    kw = dict(w.operator_kwargs())
    kw["n_t"] = n_steps + 1
    L = w.n * w.h
    op = WaveOperator(Domain((w.n, w.n), ((0.0, L), (0.0, L)), axes=("x", "z")), torch.tensor(w.sources[:n_shots]),
                      torch.tensor(w.receivers), grad_mode="autograd", **kw)
    c = torch.tensor(w.c, dtype=torch.float32, requires_grad=True)
    t0 = time.perf_counter()
    (0.5 * op({"c": c}).square().sum()).backward()
    t = time.perf_counter() - t0
    per_shot_full = t / n_shots * (w.n_steps / n_steps)
    return {"value": 1.0 / per_shot_full, "unit": UNIT, "cores": torch.get_num_threads(), "kind": "reference",
            "sample": f"nefi.physics.wave.WaveOperator (torch {torch.__version__}, CPU) forward + autograd gradient, "
                      f"{n_shots} shots x {n_steps} of {w.n_steps} steps, float32; measured {t:.2f} s, "
                      f"extrapolated linearly in shots and steps",
            "sample_s": t, "gcell_updates_per_s": 2 * w.padded_cells() * n_steps * n_shots / t / 1e9}


def run_reference(args) -> None:
    """The reference arm: the CPU restatement of the reference's algorithm (the float32 C oracle, OpenMP
    over shots on every host thread) timed on a bounded sample of the same workload per step: all of
    the workload's shots for the first REF_SAMPLE_STEPS leapfrog steps, forward and adjoint. Each step
    costs the same (fixed grid, fixed stencil), so ``value`` extrapolates the sample linearly in steps
    to the full gradient; ``ms_per_step`` is the measured time of one sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = make_workload(args)
    S = len(w.sources)
    vals, secs, info = [], [], {}
    for i in range(args.warmup + args.steps):
        v, info = cpu_sample(w, n_shots=S, n_steps=REF_SAMPLE_STEPS)
        if i >= args.warmup:
            vals.append(v)
            secs.append(info["seconds"])
    v = statistics.median(vals)
    sample_ms = 1000.0 * statistics.median(secs)
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": sample_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded)", "config": {**workload_desc(w), "parallelism": "cpu threads"},
           "sample": {"what": info["sample"], "measured_ms_per_sample": sample_ms,
                      "extrapolation": f"value = {S} shots / (sample time x {w.n_steps} / {info['steps']} steps)"},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"], "kind": "port",
                            "sample": info["sample"]},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "gcell_updates_per_s": info["gcell_updates_per_s"]}
    ref = reference_torch_sample(w)
    if ref is not None:
        out["cpu_baseline"]["reference_torch"] = ref
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------------------------------------
# the GPU arm
# ------------------------------------------------------------------------------------------------
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="fwi_512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="fwi_512: skip the batched and 2048^2 checkpointed measurements of the same line")
    ap.add_argument("--n-steps", type=int, default=None, help="override the leapfrog steps (profiling cases)")
    ap.add_argument("--shots", type=int, default=None, help="override the shots per GPU (profiling cases)")
    ap.add_argument("--problems", type=int, default=64, help="fwi_batch: problems in the batch")
    ap.add_argument("--grad-mode", default="autograd", choices=("autograd", "checkpoint"),
                    help="autograd keeps the full history when it fits, else checkpoints")
    ap.add_argument("--snapshot", default="exact", choices=("exact", "delta16", "fixed16", "fp16", "bf16"))
    ap.add_argument("--checkpoint-every", type=int, default=None)
    ap.add_argument("--absorbing", default=None, choices=("sponge", "pml", "cerjan", "none"),
                    help="override the workload's absorbing layer (fwi workloads)")
    ap.add_argument("--tuning", default=None,
                    help="launch shapes vz,rx,shots_per_cta,adj_vz,adj_rx,adj_shots_per_cta[,depth] (0: default)")
    ap.add_argument("--depth", type=int, default=0, choices=(0, 1, 2),
                    help="fwi workloads: forward steps per launch (0: the library default)")
    ap.add_argument("--pat-n", type=int, default=256, help="pat_256: grid edge (profiling cases)")
    ap.add_argument("--fd-directions", type=int, default=8,
                    help="central finite-difference checks of the float64 gradient (0: none)")
    ap.add_argument("--accuracy-shots", type=int, default=None,
                    help="shots of the float64 accuracy check (all by default)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "fwi_batch":
        run_batch(args)
        return
    if args.workload == "pat_256":
        run_pat(args)
        return
    if args.workload == "datagen_512x2":
        run_datagen(args)
        return
    if args.workload == "misfit_2048":
        run_misfit(args)
        return

    import torch.distributed as dist

    from nefi_b200 import WaveOperatorB200, _lib, workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    w = make_workload(args)
    okw = w.operator_kwargs()
    if args.absorbing:
        okw["absorbing"] = args.absorbing
    op = WaveOperatorB200(w.domain, w.sources, w.receivers, grad_mode=args.grad_mode, snapshot=args.snapshot,
                          checkpoint_every=args.checkpoint_every, **okw)
    if args.depth:
        op.tuning = (0, 0, 0, 0, 0, 0, args.depth)
    if args.tuning:
        t = [int(v) for v in args.tuning.split(",")]
        op.tuning = tuple(t + [args.depth or 0] * (7 - len(t)))
    c = torch.tensor(w.c, dtype=torch.float32, device=dev)
    # observed data: traces of a smoothed model (the misfit of a typical early FWI iteration)
    with torch.no_grad():
        c_true = torch.tensor(w.c, dtype=torch.float32, device=dev)
        d = op({"c": torch.nn.functional.avg_pool2d(c_true[None, None], 9, 1, 4,
                                                    count_include_pad=False)[0, 0].contiguous()})
    flush = torch.empty(64 * 2**20, dtype=torch.float32, device=dev)
    lib = _lib.load()

    # the timed step: the whole gradient (media, forward sweep, misfit, adjoint sweep, float64
    # reduction) recorded once as a CUDA graph and replayed, so no host work sits inside the timed
    # region; under torchrun the gradient and the misfit are then summed over the ranks
    graph = op.gradient_graph(c, d, events=True)

    def step():
        graph.replay()
        if world > 1:  # the float64 gradient and the scalar misfit summed over the ranks' shots
            dist.all_reduce(graph.grad)
            dist.all_reduce(graph.loss)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    sampler = ClockSampler(dev.index if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    times, fwd_ms, adj_ms = [], [], []
    ev = None
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        ev = graph.events
        fwd_ms.append(ev["fwd0"].elapsed_time(ev["fwd1"]))
        adj_ms.append(ev["adj0"].elapsed_time(ev["adj1"]))
    torch.cuda.synchronize()
    graph.check()  # encoded snapshots: raises if a decode of the replays met a non-finite value
    if world > 1:
        dist.barrier()
    launches = graph.launches * args.steps
    clocks = sampler.stop()
    total_ms = sum(times)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t)
    S = len(w.sources)
    ms_per_step = total_ms / args.steps
    value = S * world / (ms_per_step / 1000.0)
    cells = w.padded_cells()
    gcells = 2 * cells * w.n_steps * S * world / (ms_per_step / 1000.0) / 1e9
    graph.release()
    del graph, ev
    gc.collect()  # the graph's private memory pool returns to the driver only once nothing holds it
    torch.cuda.empty_cache()

    # roofline of the dominant stencil kernel: 16 B per cell-update, per launch = cells * shots; the
    # kernels' time is the CUDA-event time of their sweeps inside the timed replays, per step
    peak, peak_kind = peaks()
    alg_bytes = 16.0 * cells * S
    fwd_launch_ms = statistics.median(fwd_ms) / w.n_steps
    adj_launch_ms = statistics.median(adj_ms) / w.n_steps
    kern = "adj2d" if adj_launch_ms >= fwd_launch_ms else "fwd2d"
    launch_ms = max(adj_launch_ms, fwd_launch_ms)
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        tj = json.loads(tf.read_text())
        if kern in tj:
            traffic = tj[kern]["bytes_per_launch_full"]
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": kern, "peak_source": peak_kind,
                "traffic_source": "profiles/traffic.json: one cold-cache ncu capture of a 100-step case, "
                                  "bytes per launch scaled to this workload; not this run's traffic",
                "algorithmic_bytes_per_launch": alg_bytes,
                "per_kernel_GBps": {"fwd2d": alg_bytes / (fwd_launch_ms * 1e-3) / 1e9,
                                    "adj2d_with_injection": alg_bytes / (adj_launch_ms * 1e-3) / 1e9}}

    # end to end through the drop-in call a NEFI solver makes (nefi/physics/wave.py:742-750): c and
    # the observed traces from pinned host memory, traces = op({"c": c}), the misfit
    # 1/2 ||traces - d||^2 in torch, loss.backward() through the autograd function, then the
    # gradient and the loss back to the host
    c_h = c.cpu().pin_memory()
    d_h = d.cpu().pin_memory()
    g_h = torch.empty(c.shape, dtype=torch.float32).pin_memory()
    l_h = torch.empty((), dtype=torch.float64).pin_memory()
    e2e_ms, e2e_storage, e2e_host = [], [], []
    gc.collect()  # Python's collector stays out of the timed calls (it can stall the host for tens of ms)
    gc.disable()
    for i in range(2 + args.steps):  # two untimed passes: the pinned copies' first use, allocator growth
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t0 = time.perf_counter()
        cd = c_h.to(dev, non_blocking=True).requires_grad_(True)
        dd = d_h.to(dev, non_blocking=True)
        loss = 0.5 * (op({"c": cd}) - dd).double().square().sum()
        t1 = time.perf_counter()
        loss.backward()
        t2 = time.perf_counter()
        g = cd.grad
        if world > 1:
            dist.all_reduce(g)
            dist.all_reduce(loss)
        g_h.copy_(g, non_blocking=True)
        l_h.copy_(loss.detach(), non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        if i > 1:
            e2e_ms.append(e0.elapsed_time(e1))
            e2e_storage.append(op.last_storage[0] if op.last_storage else None)
            e2e_host.append([round((t1 - t0) * 1e3, 1), round((t2 - t1) * 1e3, 1)])
        del cd, dd, loss, g
    e2e_total = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_total], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t)
    e2e_val = S * world / (e2e_total / len(e2e_ms) / 1000.0)
    h2d = c_h.numel() * c_h.element_size() + d_h.numel() * d_h.element_size()
    d2h = g_h.numel() * g_h.element_size() + 8

    # the same end to end through this package's own gradient call (misfit_gradient: no traces
    # materialised for torch, float64 gradient)
    g64_h = torch.empty(c.shape, dtype=torch.float64).pin_memory()
    mg_ms = []
    for i in range(2 + args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        loss, g = op.misfit_gradient(c_h.to(dev, non_blocking=True), d_h.to(dev, non_blocking=True))
        if world > 1:
            dist.all_reduce(g)
            dist.all_reduce(loss)
        g64_h.copy_(g, non_blocking=True)
        l_h.copy_(loss, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        if i > 1:
            mg_ms.append(e0.elapsed_time(e1))
        del loss, g
    gc.enable()
    mg_total = sum(mg_ms)
    if world > 1:
        t = torch.tensor([mg_total], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mg_total = float(t)
    mg_val = S * world / (mg_total / len(mg_ms) / 1000.0)

    from nefi_b200.plan import plan_storage

    mode = plan_storage(op._plan(dev, torch.float32), len(w.sources), op.n_steps, op.grad_mode,
                        op.checkpoint_every, op.snapshot, op._budget(dev))
    storage = ("full history in HBM" if mode[0] == "history" else
               f"checkpointed every {mode[1]} steps with {args.snapshot} snapshots")
    accuracy = None
    if not args.no_accuracy and rank == 0:
        # float32 gradient against a float64 device run of the same step (checkpointed, exact
        # snapshots), over the first --accuracy-shots shots (all by default)
        na = args.accuracy_shots or len(w.sources)
        kw = okw
        op32 = WaveOperatorB200(w.domain, w.sources[:na], w.receivers, grad_mode=args.grad_mode,
                                snapshot=args.snapshot, checkpoint_every=args.checkpoint_every, **kw)
        _, g32 = op32.misfit_gradient(c, d[:na])
        del op32
        op64 = WaveOperatorB200(w.domain, w.sources[:na], w.receivers, grad_mode="checkpoint", **kw)
        _, g64 = op64.misfit_gradient(c.double(), d[:na].double())
        accuracy = {"grad_rel_l2_fp32_vs_fp64": float((g32 - g64).norm() / g64.norm()), "shots": na,
                    "fp32_storage": f"{args.grad_mode}, {args.snapshot} snapshots",
                    "fixed_cotangent": fixed_cotangent_error(op64, WaveOperatorB200(
                        w.domain, w.sources[:na], w.receivers, grad_mode=args.grad_mode, snapshot=args.snapshot,
                        checkpoint_every=args.checkpoint_every, **kw), c, d[:na]),
                    "note": "grad_rel_l2_fp32_vs_fp64: each precision's own misfit gradient (its own residual); "
                            "fixed_cotangent: the float32 adjoint given the float64 residual"}
        if args.fd_directions > 0:
            # central differences of the float64 misfit along seeded unit directions, step scaled to
            # ||c||, against the float64 gradient's directional derivative
            c64, d64 = c.double(), d[:na].double()
            gen = torch.Generator(device=dev).manual_seed(2)
            eps = 1e-7 * float(c64.norm())
            errs = []
            with torch.no_grad():
                def misfit(cc):
                    return 0.5 * float((op64({"c": cc}) - d64).square().sum())
                for _ in range(args.fd_directions):
                    u = torch.randn(c64.shape, generator=gen, device=dev, dtype=torch.float64)
                    u /= u.norm()
                    fd = (misfit(c64 + eps * u) - misfit(c64 - eps * u)) / (2 * eps)
                    ad = float((g64 * u).sum())
                    errs.append(abs(fd - ad) / max(abs(ad), 1e-300))
            accuracy["fd_check"] = {"directions": args.fd_directions, "eps": eps, "max_rel_err": max(errs),
                                    "median_rel_err": statistics.median(errs), "dtype": "f64"}
        del op64

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, info = cpu_sample(w)
        cpu = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": "port", "sample": info["sample"],
               "gcell_updates_per_s": info["gcell_updates_per_s"]}

    # the north-star method under the same clock: the uneven batch (batched, checkpointed, 16-bit
    # snapshots, graph-replayed) and the large configuration (checkpointed, 16-bit snapshots), each
    # with its own roofline, accuracy against float64 and clocks; one GPU, default workload only
    extras = {}
    absorbing = op.absorbing
    if world == 1 and args.workload == "fwi_512" and not args.no_extras and not args.n_steps:
        from nefi_b200 import workloads as _wl

        op._plans.clear()  # the headline operator's device tables, so the next measurements have the device
        torch.cuda.empty_cache()
        extras["batched"] = measure_batch(dev, 1, 0, 64, steps=2, warmup=0, snapshot="delta16",
                                          with_plain=True, with_e2e=False, accuracy_problems=0 if args.no_accuracy else 4)
        extras["checkpointed_2048"] = measure_checkpointed(dev, _wl.fwi_2048(), snapshot="delta16", steps=1, warmup=1,
                                                           accuracy_shots=0 if args.no_accuracy else 4)

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded layered model; observed data from a smoothed model)",
               "config": {**workload_desc(w, storage, absorbing),
                          "method": f"plain (per-step launches replayed from one CUDA graph, {storage})",
                          "tuning": list(op.tuning) if getattr(op, "tuning", None) else "library defaults",
                          "parallelism": f"shots sharded over {world} GPU(s), fp64 gradient and loss all-reduce"},
               "gcell_updates_per_s": gcells, "roofline": roofline, "cpu_baseline": cpu,
               "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "call": "traces = op({'c': c}); loss = 1/2 ||traces - d||^2 (torch); loss.backward()",
                       "ms_each": e2e_ms, "storage_each": e2e_storage,
                       "python_gc": "collected before and disabled during the timed calls",
                       "host_ms_each": {"forward_and_loss": [h[0] for h in e2e_host],
                                        "backward": [h[1] for h in e2e_host]}},
               "e2e_misfit_gradient": {"value": mg_val, "unit": UNIT, "h2d_bytes_per_step": h2d,
                                       "d2h_bytes_per_step": g64_h.numel() * 8 + 8,
                                       "call": "op.misfit_gradient(c, d)", "ms_each": mg_ms},
               "clocks": clocks, "gpu_launches": int(launches), "accuracy": accuracy, **extras}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
