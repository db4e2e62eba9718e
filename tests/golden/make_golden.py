"""Generate golden vectors for the wave propagator by running the reference NEFI package itself.

Run where the reference checkout is available (it is not needed anywhere else), naming it by
argument or by the NEFI_REFERENCE environment variable:

    python tests/golden/make_golden.py /path/to/reference [case-name-prefix ...]
    NEFI_REFERENCE=/path/to/reference python tests/golden/make_golden.py - [case-name-prefix ...]

With name prefixes only the matching cases are written (every case is seeded on its own, so a
subset reproduces the same fixtures as a full run).

Every case stores its inputs, the operator arguments (JSON) and the reference's outputs in float64
and float32: traces of ``op(fields)`` and the gradient of ``sum(traces * g)`` for a seeded
cotangent ``g``, taken with ``torch.autograd`` through the reference's unrolled loop (grad_mode
"autograd"). For the photoacoustic operator the gradient w.r.t. the (frozen) sound speed is taken
through the reference's own internals, the same calls its ``simulate`` makes
(nefi/physics/wave.py:840-867).
"""

from __future__ import annotations

import json
import math
import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
_arg = sys.argv[1] if len(sys.argv) > 1 else "-"
if _arg == "-" and not os.environ.get("NEFI_REFERENCE"):
    sys.exit("usage: make_golden.py /path/to/reference [case-name-prefix ...] "
             "(or '-' with NEFI_REFERENCE set to the reference checkout)")
REF = Path(os.environ["NEFI_REFERENCE"] if _arg == "-" else _arg)
ONLY = tuple(sys.argv[2:])
sys.path.insert(0, str(REF))

from nefi.domain import Domain  # noqa: E402
from nefi.physics.timestep import run_timestepping  # noqa: E402
from nefi.physics.wave import WaveInitialConditionOperator, WaveOperator, laplacian, time_reversal  # noqa: E402

F64, F32 = torch.float64, torch.float32


def cotangent(shape, seed):
    """Seeded trace cotangent g (regenerated by the tests from the stored seed)."""
    return torch.randn(tuple(shape), generator=torch.Generator().manual_seed(seed), dtype=F64)


def fwi_case(name, shape, extent, sources, receivers, c, kw, seed, rec_stride=1):
    if not wanted(name):
        return
    dom = Domain(shape, extent)
    out = {"kind": "fwi", "shape": list(shape), "extent": [list(e) for e in extent],
           "sources": np.asarray(sources, dtype=np.float64), "receivers": np.asarray(receivers, dtype=np.float64),
           "c": c.numpy(), "kw": kw, "seed": seed, "rec_stride": rec_stride}
    for dt, tag in ((F64, "f64"), (F32, "f32")):
        op = WaveOperator(dom, sources, receivers, grad_mode="autograd", **kw)
        x = c.to(dt).clone().requires_grad_(True)
        tr = op({"c": x})
        gtr = cotangent(tr.shape, seed)
        (gc,) = torch.autograd.grad((tr * gtr.to(dt)).sum(), x)
        out[f"traces_{tag}"] = tr.detach()[:, ::rec_stride].numpy()
        out[f"grad_c_{tag}"] = gc.numpy()
        out["meta"] = {"substeps": op.substeps, "n_steps": op.n_steps, "dt": op.dt,
                       "padded": list(op.grid.padded_shape), "n_abs": list(op.grid.n_abs)}
    save(name, out)


def pat_case(name, shape, extent, receivers, p0, c, kw, seed):
    if not wanted(name):
        return
    dom = Domain(shape, extent)
    out = {"kind": "pat", "shape": list(shape), "extent": [list(e) for e in extent],
           "receivers": np.asarray(receivers, dtype=np.float64), "p0": p0.numpy(), "c": c.numpy(), "kw": kw,
           "seed": seed, "rec_stride": 1}
    for dt, tag in ((F64, "f64"), (F32, "f32")):
        op = WaveInitialConditionOperator(dom, receivers, c=c, grad_mode="autograd", **kw)
        x = p0.to(dt).clone().requires_grad_(True)
        tr = op({"p0": x})
        gtr = cotangent(tr.shape, seed)
        (gp,) = torch.autograd.grad((tr * gtr.to(dt)).sum(), x)
        out[f"traces_{tag}"] = tr.detach().numpy()
        out[f"grad_p0_{tag}"] = gp.numpy()
        # gradient w.r.t. the sound speed through the reference's own step function; like the
        # operator (nefi/physics/wave.py:814-820) c2dt2 is formed in float64 and then cast
        st = op._static(torch.device("cpu"), dt)
        cl = c.clone().requires_grad_(True)
        c2dt2 = (op.grid.pad(cl, "replicate") ** 2 * op.dt**2).to(dt)
        p0p = op.grid.pad(p0.to(dt).reshape(-1, *shape), "zeros")
        pm1 = p0p + 0.5 * c2dt2 * laplacian(p0p, op.grid.spacing, op.order, st["kernel"])
        ridx, rw = st["rec_idx"], st["rec_w"]
        d = len(shape)

        def observe(s, n):
            return (s[1].reshape(*s[1].shape[:-d], -1)[..., ridx] * rw).sum(-1)

        _, obs = run_timestepping(op._step_fn(st, None), op._initial_state(pm1, p0p), (c2dt2,),
                                  op.n_steps, op.dt, observe, record=op.record)
        yc = torch.stack(obs, -1).reshape(tr.shape)
        assert float((yc.detach() - tr.detach()).abs().max()) == 0.0
        (gc,) = torch.autograd.grad((yc * gtr.to(dt)).sum(), cl)
        out[f"grad_c_{tag}"] = gc.numpy()
        out["meta"] = {"substeps": op.substeps, "n_steps": op.n_steps, "dt": op.dt,
                       "padded": list(op.grid.padded_shape), "n_abs": list(op.grid.n_abs)}
    save(name, out)


def tr_case(name, shape, extent, receivers, traces, kw, seed):
    """time_reversal(mode="dirichlet") of given traces (nefi/physics/wave.py:878-968)."""
    if not wanted(name):
        return
    dom = Domain(shape, extent)
    kw = dict(kw)
    c = kw.pop("c")
    c = c if isinstance(c, torch.Tensor) else torch.full(tuple(shape), float(c), dtype=F64)
    out = {"kind": "tr", "shape": list(shape), "extent": [list(e) for e in extent],
           "receivers": np.asarray(receivers, dtype=np.float64), "traces": traces.numpy(), "c": c.numpy(),
           "kw": kw, "seed": seed, "rec_stride": 1}
    for dt, tag in ((F64, "f64"), (F32, "f32")):
        p0 = time_reversal(traces.to(dt), dom, receivers, mode="dirichlet", c=c, **kw)
        out[f"p0_{tag}"] = p0.numpy()
    save(name, out)


def gen_case(name, shape, extent, sources, receivers, c_fine, kw, factor):
    """FP64 data generation as ``DataGenerator.clean`` does it (nefi/bench/base.py:74-90): an operator
    built on the native grid, moved to float64, called through ``at_resolution`` with the ground truth
    on the ``factor``-times refined grid (the 2x-supersampled wave_fwi generator,
    nefi/instances/wave_fwi/__init__.py:248-260)."""
    if not wanted(name):
        return
    dom = Domain(shape, extent)
    op = WaveOperator(dom, sources, receivers, **kw).to(dtype=F64)
    fine = tuple(int(s) * factor for s in shape)
    with torch.no_grad():
        tr = op.at_resolution(fine)({"c": c_fine.to(F64)})
    out = {"kind": "gen", "shape": list(shape), "fine": list(fine), "extent": [list(e) for e in extent],
           "sources": np.asarray(sources, dtype=np.float64), "receivers": np.asarray(receivers, dtype=np.float64),
           "c": c_fine.numpy(), "kw": kw, "seed": 0, "rec_stride": 1, "traces_f64": tr.numpy()}
    save(name, out)


def misfit_case(name, n_rows, n_t, dt, kw, seed, mask_rows=None, sensor=None):
    """The reference's trace misfit: ``BandLimitedMSE(**kw).forward(ctx)`` (wave_fwi/losses.py:51-86)
    and its gradient w.r.t. the prediction by autograd, ``lowpass`` of the prediction, and -- with
    ``sensor`` -- ``gaussian_lowpass`` (photoacoustic3d/sensor.py:24-38) of the prediction and the
    gradient of the MSE of the sensor-filtered prediction (nefi/losses/data.py:46-52)."""
    if not wanted(name):
        return
    from nefi.instances.photoacoustic3d.sensor import gaussian_lowpass
    from nefi.instances.wave_fwi.losses import BandLimitedMSE, lowpass
    from nefi.losses.data import MSE
    from nefi.measurement import Measurement

    g = torch.Generator().manual_seed(seed)
    t = torch.arange(n_t, dtype=F64) * dt
    f = 1.0 / (8 * dt) * (0.5 + torch.rand(n_rows, 1, generator=g, dtype=F64))
    obs = torch.sin(2 * math.pi * f * t) * torch.exp(-t / (n_t * dt)) + 0.3 * torch.randn(n_rows, n_t, generator=g, dtype=F64)
    pred = obs + 0.5 * torch.randn(n_rows, n_t, generator=g, dtype=F64)
    mask = None
    if mask_rows is not None:
        mask = torch.ones(n_rows, 1, dtype=F64)
        mask[mask_rows] = 0.0
    out = {"kind": "misfit", "pred": pred.numpy(), "obs": obs.numpy(), "dt": dt, "kw": kw, "seed": seed,
           "sensor": sensor}
    if mask is not None:
        out["mask"] = mask.numpy()

    class Ctx:  # the two attributes a data loss reads (nefi/losses/base.py:26-38)
        def __init__(self, p, m):
            self.pred, self.obs = p, m

    for dt_, tag in ((F64, "f64"), (F32, "f32")):
        x = pred.to(dt_).clone().requires_grad_(True)
        meas = Measurement(obs.to(dt_), None if mask is None else mask.to(dt_))
        loss = BandLimitedMSE(**kw).forward(Ctx(x, meas))
        (gx,) = torch.autograd.grad(loss, x)
        out[f"loss_{tag}"] = np.array(float(loss))
        out[f"grad_{tag}"] = gx.numpy()
        if kw.get("f_max") is not None:
            out[f"lowpass_{tag}"] = lowpass(pred.to(dt_), dt, kw["f_max"], kw.get("taper", 0.3)).numpy()
        if sensor is not None:
            x = pred.to(dt_).clone().requires_grad_(True)
            y = gaussian_lowpass(x, dt, sensor)
            loss = MSE().forward(Ctx(y, meas))
            (gx,) = torch.autograd.grad(loss, x)
            out[f"sensor_{tag}"] = y.detach().numpy()
            out[f"sensor_loss_{tag}"] = np.array(float(loss))
            out[f"sensor_grad_{tag}"] = gx.numpy()
    save(name, out)


def gen_pat_case(name, shape, extent, receivers, c_coarse, p0_fine, kw, factor):
    """Photoacoustic traces through ``at_resolution`` (nefi/physics/wave.py:822-835): the operator built
    on the native grid with a known speed map, called with ``p0`` on the refined grid, so the speed is
    resampled (nefi/utils/tensor.py:35-69) before the run; float64."""
    if not wanted(name):
        return
    dom = Domain(shape, extent)
    op = WaveInitialConditionOperator(dom, receivers, c=c_coarse, **kw).to(dtype=F64)
    fine = tuple(int(s) * factor for s in shape)
    with torch.no_grad():
        tr = op.at_resolution(fine)({"p0": p0_fine.to(F64)})
    out = {"kind": "genpat", "shape": list(shape), "fine": list(fine), "extent": [list(e) for e in extent],
           "receivers": np.asarray(receivers, dtype=np.float64), "c": c_coarse.numpy(), "p0": p0_fine.numpy(),
           "kw": kw, "seed": 0, "rec_stride": 1, "traces_f64": tr.numpy()}
    save(name, out)


def wanted(name):
    return not ONLY or name.startswith(ONLY)


def save(name, out):
    arrays = {k: v for k, v in out.items() if isinstance(v, np.ndarray)}
    meta = {k: v for k, v in out.items() if not isinstance(v, np.ndarray)}
    for k, v in list(arrays.items()):
        if v.dtype == np.float64 and k.endswith("_f32"):
            arrays[k] = v.astype(np.float32)
    np.savez_compressed(HERE / f"{name}.npz", meta=json.dumps(meta), **arrays)
    print(name, {k: v.shape for k, v in arrays.items()}, meta.get("meta"))


def main():
    torch.manual_seed(0)
    # small FWI cases, 2-D (the geometry of the reference's own adjoint checks)
    c = (2.0 + 0.2 * torch.randn(20, 24, dtype=F64)).clamp(1.6, 2.4)
    src = [[0.3, 0.2], [0.6, 0.5]]
    rec = [[0.8, y] for y in (0.2, 0.5, 0.9)]
    base = dict(n_t=30, dt_obs=0.012, f0=6.0, c_max=2.5)
    ext = ((0.0, 1.0), (0.0, 1.2))
    fwi_case("fwi_o4_sponge", (20, 24), ext, src, rec, c, {**base, "order": 4, "absorbing": "sponge",
                                                             "absorb_width": 0.2}, 1)
    fwi_case("fwi_o2_none", (20, 24), ext, src, rec, c, {**base, "order": 2, "absorbing": "none"}, 2)
    fwi_case("fwi_o4_cerjan", (20, 24), ext, src, rec, c, {**base, "order": 4, "absorbing": "cerjan",
                                                             "absorb_width": 0.2, "cerjan_gamma": 0.5}, 3)
    c2 = (2.0 + 0.2 * torch.randn(18, 30, dtype=F64)).clamp(1.6, 2.4)
    fwi_case("fwi_o2_sponge_aniso", (18, 30), ((0.0, 0.9), (0.0, 1.2)), [[0.45, 0.1]],
             [[0.1 + 0.1 * i, 1.0] for i in range(7)], c2,
             {**base, "n_t": 25, "order": 2, "absorbing": "sponge", "absorb_width": 0.16, "courant": 0.8}, 4)
    # the plain 128^2 FWI workload: h = 10 m, 2000 m/s + two +-300 m/s Gaussian anomalies (sigma 8 cells),
    # 20-cell sponge, one 15 Hz Ricker at top centre, 128 receivers on row 2, 1000 steps at CFL 0.4.
    n, h = 128, 10.0
    rng = torch.Generator().manual_seed(0)
    xs = (torch.arange(n, dtype=F64) + 0.5) * h
    X, Z = torch.meshgrid(xs, xs, indexing="ij")
    cc = torch.full((n, n), 2000.0, dtype=F64)
    for s in (1.0, -1.0):
        ctr = torch.rand(2, generator=rng, dtype=F64) * n * h * 0.5 + n * h * 0.25
        cc = cc + s * 300.0 * torch.exp(-((X - ctr[0]) ** 2 + (Z - ctr[1]) ** 2) / (2 * (8 * h) ** 2))
    cmax = float(cc.max())
    dt = 0.4 * h / cmax
    fwi_case("cfg1_128_o4_sponge", (n, n), ((0.0, n * h), (0.0, n * h)), [[n * h / 2, 1.5 * h]],
             [[(i + 0.5) * h, 2.5 * h] for i in range(n)], cc,
             dict(n_t=1001, dt_obs=dt, f0=15.0, c_max=cmax, order=4, absorbing="sponge",
                  absorb_width=20 * h, courant=1.0), 5, rec_stride=4)
    # photoacoustic, 2-D ring of receivers, known heterogeneous speed
    torch.manual_seed(1)
    n2 = 24
    th = 2 * math.pi * torch.arange(32, dtype=F64) / 32
    ring = torch.stack([0.85 * torch.cos(th), 0.85 * torch.sin(th)], 1)
    p0 = torch.rand(2, n2, n2, dtype=F64)
    cpat = 1.0 + 0.05 * torch.rand(n2, n2, dtype=F64)
    pat_case("pat2d_o4_sponge", (n2, n2), ((-1.0, 1.0), (-1.0, 1.0)), ring, p0, cpat,
             dict(n_t=50, dt_obs=0.03, order=4, absorbing="sponge", absorb_width=0.25), 6)
    pat_case("pat2d_o2_cerjan", (n2, n2), ((-1.0, 1.0), (-1.0, 1.0)), ring, p0[0], cpat,
             dict(n_t=40, dt_obs=0.03, order=2, absorbing="cerjan", absorb_width=0.25), 7)
    # photoacoustic, 3-D slab with a planar sensor array on the top face
    xs3 = (torch.arange(4, dtype=F64) + 0.5) * 0.75
    Xs, Ys = torch.meshgrid(xs3, xs3, indexing="ij")
    sens = torch.stack([Xs.ravel(), Ys.ravel(), torch.zeros(16, dtype=F64)], -1)
    p03 = torch.rand(12, 12, 8, dtype=F64)
    c3 = 1.5 * (1.0 + 0.05 * torch.rand(12, 12, 8, dtype=F64))
    pat_case("pat3d_o2_sponge", (12, 12, 8), ((0.0, 3.0), (0.0, 3.0), (0.0, 2.0)), sens, p03, c3,
             dict(n_t=30, dt_obs=0.1, order=2, absorbing="sponge", absorb_width=0.75), 8)
    sens_in = sens * 0.8
    sens_in[:, 2] = 0.125  # first cell centre: without a layer the sensors must sit inside the grid
    pat_case("pat3d_o4_none", (10, 9, 8), ((0.0, 2.5), (0.0, 2.25), (0.0, 2.0)), sens_in, p03[:10, :9],
             c3[:10, :9], dict(n_t=20, dt_obs=0.08, order=4, absorbing="none"), 9)
    # 2-D PML (the reference's default layer), FWI and photoacoustic, same geometries as above
    fwi_case("fwi_o4_pml", (20, 24), ext, src, rec, c, {**base, "order": 4, "absorbing": "pml",
                                                         "absorb_width": 0.2}, 10)
    fwi_case("fwi_o2_pml_aniso", (18, 30), ((0.0, 0.9), (0.0, 1.2)), [[0.45, 0.1]],
             [[0.1 + 0.1 * i, 1.0] for i in range(7)], c2,
             {**base, "n_t": 25, "order": 2, "absorbing": "pml", "absorb_width": 0.16, "courant": 0.8}, 11)
    pat_case("pat2d_o4_pml", (n2, n2), ((-1.0, 1.0), (-1.0, 1.0)), ring, p0, cpat,
             dict(n_t=50, dt_obs=0.03, order=4, absorbing="pml", absorb_width=0.25), 12)
    # classical PAT baseline: Dirichlet time reversal of smooth seeded traces (2 substeps per sample)
    gtr = torch.Generator().manual_seed(13)
    tt = torch.linspace(0.0, 1.0, 40, dtype=F64)
    trc = torch.stack([torch.sin(6.0 * tt + 2 * math.pi * torch.rand(1, generator=gtr, dtype=F64))
                       * torch.exp(-3.0 * tt) for _ in range(32)])
    tr_case("tr2d_o4_pml", (n2, n2), ((-1.0, 1.0), (-1.0, 1.0)), ring, trc,
            dict(dt_obs=0.03, c=cpat, order=4, absorbing="pml", absorb_width=0.25), 13)
    tr_case("tr2d_o2_sponge", (n2, n2), ((-1.0, 1.0), (-1.0, 1.0)), ring, trc,
            dict(dt_obs=0.03, c=1.0, order=2, absorbing="sponge", absorb_width=0.25, courant=0.8), 14)
    tr3 = torch.stack([torch.sin(5.0 * tt[:24] + 0.3 * k) * torch.exp(-2.0 * tt[:24]) for k in range(16)])
    tr_case("tr3d_o2_sponge", (12, 12, 8), ((0.0, 3.0), (0.0, 3.0), (0.0, 2.0)), sens, tr3,
            dict(dt_obs=0.1, c=c3, order=2, absorbing="sponge", absorb_width=0.75), 15)
    # FP64 data generation at 2x supersampling through at_resolution (order-4 generator, both layers)
    cf = (2.0 + 0.2 * torch.randn(40, 48, generator=torch.Generator().manual_seed(16), dtype=F64)).clamp(1.6, 2.4)
    cf = torch.nn.functional.avg_pool2d(cf[None, None], 3, 1, 1, count_include_pad=False)[0, 0]
    gen_case("gen2x_o4_pml", (20, 24), ext, src, rec, cf, {**base, "order": 4, "absorbing": "pml",
                                                            "absorb_width": 0.2}, 2)
    gen_case("gen2x_o4_sponge", (20, 24), ext, src, rec, cf, {**base, "order": 4, "absorbing": "sponge",
                                                               "absorb_width": 0.2}, 2)
    # trace misfit: band-limited relative MSE (with a muted-trace mask), absolute, unfiltered; sensor response
    misfit_case("misfit_bl_rel", 6, 120, 0.004, {"f_max": 30.0, "dt": 0.004, "taper": 0.3, "relative": True}, 17)
    misfit_case("misfit_bl_mask", 7, 333, 0.002, {"f_max": 45.0, "dt": 0.002, "taper": 0.5, "relative": True}, 18,
                mask_rows=[1, 4], sensor=60.0)
    misfit_case("misfit_bl_abs", 5, 1001, 0.001, {"f_max": 25.0, "dt": 0.001, "taper": 0.2, "relative": False}, 19,
                sensor=80.0)
    misfit_case("misfit_plain_rel", 4, 64, 0.01, {"f_max": None, "dt": 0.01, "relative": True}, 20, mask_rows=[2])
    # a brick-wall window (taper 0) whose cutoff falls on an rfft bin up to rounding (f_108 of 540 bins)
    misfit_case("misfit_brick", 3, 257, 0.002, {"f_max": 100.0, "dt": 0.002, "taper": 0.0, "relative": True}, 21)

    # photoacoustic traces through at_resolution: a 2-D speed map resampled to the refined grid
    gp = torch.Generator().manual_seed(22)
    cpc = 1.0 + 0.05 * torch.rand(n2, n2, generator=gp, dtype=F64)
    p0f = torch.rand(2 * n2, 2 * n2, generator=gp, dtype=F64)
    gen_pat_case("genpat2x_o4_sponge", (n2, n2), ((-1.0, 1.0), (-1.0, 1.0)), ring, cpc, p0f,
                 dict(n_t=40, dt_obs=0.03, order=4, absorbing="sponge", absorb_width=0.25), 2)

    # 2-D PML on a grid whose interior holds whole step tiles, so that a propagator which sends the
    # trivial interior box through its plain step and only the layer through the PML update is
    # checked against the reference on both parts
    gb = torch.Generator().manual_seed(21)
    cb = (2.0 + 0.15 * torch.randn(56, 200, generator=gb, dtype=F64)).clamp(1.7, 2.3)
    cb = torch.nn.functional.avg_pool2d(cb[None, None], 5, 1, 2, count_include_pad=False)[0, 0]
    fwi_case("fwi_o4_pml_box", (56, 200), ((0.0, 0.56), (0.0, 2.0)), [[0.05, 0.4], [0.3, 1.5]],
             [[0.02, 0.1 + 0.09 * i] for i in range(20)] + [[0.5, 1.0]], cb,
             dict(n_t=50, dt_obs=0.004, f0=25.0, c_max=2.5, order=4, absorbing="pml", absorb_width=0.08), 23)
    # the same grid with receivers on the domain's four faces: their stencils reach the first layer
    # row or column, so a propagator that adds the interior's and the layer's cotangents in different
    # places is checked on both
    fwi_case("fwi_o4_pml_faces", (56, 200), ((0.0, 0.56), (0.0, 2.0)), [[0.05, 0.4], [0.3, 1.5]],
             [[0.02, 0.1 + 0.09 * i] for i in range(20)] + [[0.5, 1.0], [0.0, 0.77], [0.33, 0.0], [0.56, 1.3],
                                                            [0.41, 2.0]], cb,
             dict(n_t=50, dt_obs=0.004, f0=25.0, c_max=2.5, order=4, absorbing="pml", absorb_width=0.08), 23)


if __name__ == "__main__":
    main()
