"""Host-side logic on the CPU: the operators' geometry and the device tables they build reproduce the
reference's results when the kernels' semantics are replayed in numpy (tests/kernel_model.py)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import cotangent, full_trace_shape, golden_names, load_golden, rel_l2
from kernel_model import GhostModel
from nefi_b200 import WaveInitialConditionOperatorB200, WaveOperatorB200
from nefi_b200._compat import ConfigError, Domain, OperatorError, ShapeError

SMALL_FWI = [n for n in golden_names("fwi") if not n.startswith("cfg1")]
PAT = golden_names("pat")
CPU = torch.device("cpu")


def make_op(case):
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    if case["kind"] == "fwi":
        return WaveOperatorB200(dom, case["sources"], case["receivers"], grad_mode="autograd", **case["kw"])
    return WaveInitialConditionOperatorB200(dom, case["receivers"], c=torch.tensor(case["c"]),
                                            grad_mode="autograd", **case["kw"])


@pytest.mark.parametrize("name", golden_names("fwi") + golden_names("pat"))
def test_time_axis_and_padding_match_reference(name):
    case = load_golden(name)
    op = make_op(case)
    meta = case["meta"]
    assert op.substeps == meta["substeps"] and op.n_steps == meta["n_steps"]
    assert op.dt == pytest.approx(meta["dt"], rel=1e-15)
    assert list(op.grid.padded_shape) == meta["padded"] and list(op.grid.n_abs) == meta["n_abs"]


@pytest.mark.parametrize("name", SMALL_FWI)
def test_fwi_tables_reproduce_reference(name):
    case = load_golden(name)
    op = make_op(case)
    model = GhostModel(op._plan(CPU, torch.float64))
    C = model.medium(case["c"], op.dt**2)
    g = cotangent(full_trace_shape(case), case["seed"])
    tr, gC, _, _ = model.run(C, op.n_steps, op.substeps, op.n_t, list(range(op.n_sources)), grad_traces=g)
    assert rel_l2(tr, case["traces_f64"]) < 1e-12
    assert rel_l2(model.fold_grad(case["c"], op.dt**2, gC), case["grad_c_f64"]) < 1e-11


@pytest.mark.parametrize("name", PAT)
def test_pat_tables_reproduce_reference(name):
    case = load_golden(name)
    op = make_op(case)
    plan = op._plan(CPU, torch.float64)
    model = GhostModel(plan)
    d = len(case["shape"])
    p0 = case["p0"].reshape(-1, *case["shape"])
    S = p0.shape[0]
    C = np.zeros(model.F)
    c2 = op.grid.pad(torch.tensor(case["c"]), "replicate").numpy() ** 2 * op.dt**2
    C[model.I] = c2.reshape(-1)
    cur = np.zeros((S, model.F))
    padded = np.pad(p0, [(0, 0)] + [(a, a) for a in op.grid.n_abs])
    cur[:, model.I] = padded.reshape(S, -1)
    prev = np.zeros((S, model.F))
    for s in range(S):
        prev[s, model.I] = cur[s, model.I] + (0.5 * C[model.I]) * model.lap(cur[s])
    g = cotangent(full_trace_shape(case), case["seed"]).reshape(S, plan.n_rec, op.n_t)
    tr, gC, lam0, mu1 = model.run(C, op.n_steps, op.substeps, op.n_t, list(range(S)), init=(prev, cur),
                                  grad_traces=g)
    assert rel_l2(tr.reshape(case["traces_f64"].shape), case["traces_f64"]) < 1e-12
    b0 = 1.0 if (model.B is None or plan.first_b_one) else model.B
    gp = np.zeros((S, *case["shape"]))
    for s in range(S):
        lm1 = -(b0 * mu1[s])
        full = (lam0[s] + lm1)[model.I] + model.lap(0.5 * C * lm1)
        dense = full.reshape(model.P)
        sl = tuple(slice(a, a + n) for a, n in zip(op.grid.n_abs, case["shape"]))
        gp[s] = dense[sl]
        gC[s, model.I] += (0.5 * lm1[model.I]) * model.lap(cur[s])
    assert rel_l2(gp.reshape(case["grad_p0_f64"].shape), case["grad_p0_f64"]) < 1e-11
    gc = model.fold_grad(case["c"], op.dt**2, gC)
    assert rel_l2(gc, case["grad_c_f64"]) < 1e-11
    assert d in (2, 3)


def test_adjoint_table_is_cell_major_and_complete():
    case = load_golden("fwi_o4_sponge")
    plan = make_op(case)._plan(CPU, torch.float64)
    cells = plan.cell_index.numpy()
    assert np.all(np.diff(cells) > 0)
    ptr = plan.cell_ptr.numpy()
    assert ptr[0] == 0 and ptr[-1] == plan.rec_index.numel()
    # every (receiver, corner) pair appears exactly once
    pairs = sorted(zip(plan.cell_rec.numpy().tolist(), plan.cell_weight.numpy().tolist()))
    ref = sorted((r, w) for r in range(plan.n_rec) for w in plan.rec_weight[r].tolist())
    assert pairs == ref


@pytest.mark.parametrize("tuning", [(0, 0, 0), (2, 2, 1, 2, 8, 1), (4, 8, 3, 4, 2, 2), (2, 4, 16, 2, 4, 5)])
@pytest.mark.parametrize("name", ["fwi_o4_sponge", "cfg1_128_o4_sponge", "pat2d_o4_sponge"])
def test_tile_tables_partition_receivers_and_cells(name, tuning):
    """Every receiver is owned by exactly the forward tile holding its stencil corner, and every
    receiver-touched cell appears once, in its own adjoint tile, at the right local index."""
    case = load_golden(name)
    plan = make_op(case)._plan(CPU, torch.float32)
    plan.set_tuning(*tuning)
    _check_tile_tables(plan)


def _check_tile_tables(plan):
    TX, TZ = plan.tile
    assert TX == 8 * plan.tuning.rx and TZ == 32 * plan.tuning.vz
    AX, AZ = plan.adj_tile
    assert AX == 8 * plan.tuning.adj_rx and AZ == 32 * plan.tuning.adj_vz
    tz = plan.tiles_z
    rptr, rlist = plan.tile_rec_ptr.numpy(), plan.tile_rec_list.numpy()
    corner = plan.rec_corner.numpy()
    assert sorted(rlist.tolist()) == list(range(plan.n_rec))
    for t in range(len(rptr) - 1):
        for r in rlist[rptr[t]:rptr[t + 1]]:
            assert (corner[r, 0] // TX) * tz + corner[r, 1] // TZ == t
    atz = plan.adj_tiles_z
    cptr = plan.tile_cell_ptr.numpy()
    gid, local = plan.tile_cell_gid.numpy(), plan.tile_cell_local.numpy()
    cells = plan.cell_index.numpy() - plan.g.origin
    ld = plan.g.stride[0]
    # the adjoint tile grid starts at the PML's tiled box when the tables were built for it; the
    # touched cells outside the box are then listed apart, ascending, for the layer's launch
    ox, oz = plan.adj_box_corner if plan.adj_tables_box else (0, 0)
    box = plan.pml_tiled_box(AX, AZ)
    if plan.adj_tables_box:
        assert box is not None and (ox, oz) == (box[0], box[2])
        assert atz == -(-(box[3] - box[2]) // AZ) and len(cptr) - 1 == atz * -(-(box[1] - box[0]) // AX)
        off, lgid = plan.layer_cell_index.numpy(), plan.layer_cell_gid.numpy()
        assert np.all(np.diff(off) > 0)
        assert np.array_equal(off, plan.cell_index.numpy()[lgid])
        xs, zs = (off - plan.g.origin) // ld, (off - plan.g.origin) % ld
        assert not ((xs >= box[0]) & (xs < box[1]) & (zs >= box[2]) & (zs < box[3])).any()
        assert sorted(gid.tolist() + lgid.tolist()) == list(range(plan.n_cells))
    else:
        assert box is None or plan.n_cells == 0
        assert sorted(gid.tolist()) == list(range(plan.n_cells))
    for t in range(len(cptr) - 1):
        x0, z0 = ox + (t // atz) * AX, oz + (t % atz) * AZ
        for e in range(cptr[t], cptr[t + 1]):
            x, z = divmod(int(cells[gid[e]]), ld)
            assert x0 <= x < x0 + AX and z0 <= z < z0 + AZ
            assert local[e] == (x - x0) * AZ + (z - z0)


def test_tile_tables_partition_random_geometries():
    """The same invariants over seeded random grids, layers, tile shapes and receivers, including
    receivers on the outermost admissible positions (the domain's corners with a layer, the corner
    cell centres without), on cell centres and sharing cells."""
    import random

    rnd = random.Random(1234)
    for _ in range(25):
        n0, n1 = rnd.randint(8, 300), rnd.randint(8, 300)
        h = rnd.choice([0.01, 0.02, 0.005])
        ext = ((0.0, n0 * h), (0.0, n1 * h))
        width = rnd.choice([0.0, 3 * h, 20 * h])
        # without a layer a point must lie between the outermost cell centres (the reference's rule)
        a0, a1 = (0.0, 0.0) if width else (0.5 * h, 0.5 * h)
        b0, b1 = (n0 * h - a0, n1 * h - a1)
        rec = [[rnd.uniform(a0, b0), rnd.uniform(a1, b1)] for _ in range(rnd.randint(1, 40))]
        rec += [[a0, a1], [b0, b1], [a0, b1], [(0.5 + rnd.randrange(n0)) * h, 0.5 * h]]
        rec += rec[:2]  # coincident receivers
        order = rnd.choice([2, 4])
        absorbing = "none" if width == 0.0 else rnd.choice(["sponge", "pml", "cerjan"])
        op = WaveOperatorB200(Domain((n0, n1), ext), [[0.5 * n0 * h, 0.5 * n1 * h]], rec, n_t=5,
                              dt_obs=0.001, f0=10.0, c_max=2.0, order=order, absorbing=absorbing,
                              absorb_width=width)
        for dtype in (torch.float32, torch.float64):
            plan = op._plan(CPU, dtype)
            vz = [2, 4] if dtype == torch.float32 else [2]
            plan.set_tuning(rnd.choice(vz), rnd.choice([2, 4, 8]), rnd.randint(1, 5),
                            rnd.choice(vz), rnd.choice([2, 4, 8]), rnd.randint(1, 5))
            _check_tile_tables(plan)


@pytest.mark.parametrize("n_shots", [1, 3, 16, 64])
@pytest.mark.parametrize("tuning", [(0, 0, 0), (2, 4, 3, 2, 2, 2), (4, 2, 1, 4, 8, 5)])
def test_adjoint_accumulators_are_one_per_shot_group(n_shots, tuning):
    case = load_golden("fwi_o4_sponge")
    plan = make_op(case)._plan(CPU, torch.float32)
    plan.set_tuning(*tuning)
    spc = plan.tuning.adj_shots_per_cta
    assert plan.n_acc(n_shots) == -(-n_shots // spc)
    assert plan.shots_per_acc(n_shots) == spc


def test_reference_errors_are_raised_on_the_host():
    dom = Domain((16, 16), ((0.0, 1.0), (0.0, 1.0)))
    kw = dict(n_t=10, dt_obs=0.01, f0=5.0, c_max=2.5, absorbing="sponge")
    with pytest.raises(ConfigError):
        WaveOperatorB200(dom, [[0.5, 0.5]], [[0.5, 0.5]], **{**kw, "absorbing": "bogus"})
    with pytest.raises(ConfigError):
        WaveOperatorB200(dom, [[0.5, 0.5]], [[0.5, 0.5]], **{**kw, "order": 6})
    with pytest.raises(ConfigError):
        WaveOperatorB200(dom, [[0.5, 0.5]], [[0.5, 0.5]], **kw, grad_mode="other")
    with pytest.raises(ConfigError):  # outside the padded grid
        WaveOperatorB200(dom, [[5.0, 0.5]], [[0.5, 0.5]], **kw)
    op = WaveOperatorB200(dom, [[0.5, 0.5]], [[0.5, 0.5]], **kw)
    with pytest.raises(ShapeError):
        op({"c": torch.ones(8, 8, dtype=torch.float64)})
    with pytest.raises(ConfigError, match="CUDA"):  # no CPU path
        op({"c": torch.full((16, 16), 2.0, dtype=torch.float64)})
    with pytest.raises(OperatorError):
        op._check_speed(torch.full((16, 16), 3.0))
    with pytest.raises(ConfigError):
        WaveInitialConditionOperatorB200(Domain((4, 4, 4), ((0, 1),) * 3), [[0.5, 0.5, 0.5]], n_t=3,
                                         dt_obs=0.1, absorbing="pml")


def test_attributes_mirror_reference_operator():
    dom = Domain((32, 32), ((0.0, 1.0), (0.0, 1.0)))
    src = [[0.1, 0.3], [0.1, 0.5], [0.1, 0.7]]
    rec = [[0.9, y] for y in torch.linspace(0.1, 0.9, 6).tolist()]
    op = WaveOperatorB200(dom, src, rec, n_t=60, dt_obs=0.016, f0=3.0, c_max=2.5, absorb_width=0.25,
                          absorbing="sponge")
    assert op.output_shape((32, 32)) == (3, 6, 60)
    assert op.fidelity_tag == "wave-leapfrog-o4-sponge" and op.homogeneity is None
    assert op.traceable is False and op.batchable is False and op.primary == "c"
    coarse = op.at_resolution((16, 16))
    assert coarse is op.at_resolution((16, 16)) and coarse.grid.shape == (16, 16)
    assert coarse.fidelity_tag == op.fidelity_tag
    assert op.record == [j * op.substeps for j in range(60)]
    assert op.times.shape == (60,) and op.wavelet().shape == (op.n_steps,)
    pat = WaveInitialConditionOperatorB200(dom, rec, n_t=20, dt_obs=0.01, absorbing="sponge")
    assert pat.homogeneity == 1.0 and pat.fidelity_tag == "wave-leapfrog-ic-o4-sponge"
    assert pat.output_shape((32, 32)) == (6, 20)


def test_time_reversal_refuses_host_traces():
    """The baseline runs on the device only: host traces are an error, never a CPU fallback."""
    from nefi_b200 import time_reversal

    case = load_golden("tr2d_o4_pml")
    dom = Domain(tuple(case["shape"]), tuple(tuple(e) for e in case["extent"]))
    for mode in ("dirichlet", "adjoint"):
        with pytest.raises(ConfigError):
            time_reversal(torch.tensor(case["traces"]), dom, case["receivers"], dt_obs=0.03, mode=mode)


def test_filter_response_is_the_reference_window_on_a_power_of_two_circle():
    """nw_filter_response (host code) against numpy: the reference's window -> impulse response at lags
    (-n, n) -> spectrum on 2^k points, bit-reversed and divided by 2^k."""
    import ctypes as C

    import misfit_oracle as mo
    from nefi_b200 import _lib

    lib = _lib.load()
    for kind, n_t, dt, f, taper in [(0, 120, 0.004, 30.0, 0.3), (0, 333, 0.002, 45.0, 0.5), (1, 1001, 0.001, 80.0, 0.0),
                                    (0, 44, 0.01, 12.0, 0.0)]:
        k = lib.nw_filter_log2_len(n_t)
        L = 1 << k
        assert L >= 2 * n_t and k >= 6
        hp = np.zeros(L)
        assert lib.nw_filter_response(kind, n_t, C.c_double(dt), C.c_double(f), C.c_double(taper), 1, hp.ctypes.data) == 0
        if kind == 0:
            n_fft = mo.next_fast_len(2 * n_t)
            w = mo.window(n_fft, dt, f, taper)
        else:
            n_fft = 2 * n_t
            w = np.exp(-0.5 * (np.fft.rfftfreq(n_fft, d=dt) / f) ** 2)
        h = np.fft.irfft(w, n=n_fft)
        hl = np.zeros(L)
        hl[:n_t] = h[:n_t]
        hl[L - n_t + 1:] = h[n_fft - n_t + 1:]
        H = np.fft.fft(hl).real / L
        rev = np.array([int(format(p, f"0{k}b")[::-1], 2) for p in range(L)])
        assert np.abs(hp - H[rev]).max() <= 1e-13 * np.abs(H).max()
    with pytest.raises(_lib.LibraryError):
        _lib.check(lib.nw_filter_response(0, 100, C.c_double(0.0), C.c_double(10.0), C.c_double(0.3), 1,
                                          np.zeros(256).ctypes.data))


def test_misfit_refuses_host_tensors():
    from nefi_b200.misfit import TraceMisfit, lowpass

    with pytest.raises(ConfigError):
        TraceMisfit(0.01, 5.0).prepare(torch.zeros(3, 40))
    with pytest.raises(ConfigError):
        lowpass(torch.zeros(3, 40), 0.01, 5.0)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_pml_core_box_is_exactly_trivial(dtype):
    """The interior box the PML step hands to the tiled kernels: every PML term vanishes exactly on it
    (so the plain step is bitwise the PML step there), and it is the largest such box."""
    from nefi_b200.geometry import pml_coefficients
    from nefi_b200.plan import pml_core_box

    for shape, width in [((40, 56), 0.08), ((24, 24), 0.25), ((64, 33), 0.05)]:
        dom = Domain(shape, ((0.0, shape[0] * 0.01), (0.0, shape[1] * 0.01)))
        op = WaveOperatorB200(dom, [[0.05, 0.05]], [[0.02, 0.1]], n_t=10, dt_obs=0.002, f0=20.0, c_max=2.5,
                              absorbing="pml", absorb_width=width)
        co = pml_coefficients(op.grid, op.c_max, op.absorb_R, op.dt)
        cd = {k: (v.to(dtype) if torch.is_tensor(v) else [t.to(dtype) for t in v]) for k, v in co.items()}
        x0, x1, z0, z1 = pml_core_box(cd)
        P = op.grid.padded_shape
        assert 0 <= x0 <= x1 <= P[0] and 0 <= z0 <= z1 <= P[1]
        if x1 > x0:
            sl = (slice(x0, x1), slice(z0, z1))
            assert bool((cd["A"][sl] == 1).all() and (cd["B"][sl] == 1).all() and (cd["ZZ"][sl] == 0).all())
            for ax in range(2):
                lo = [slice(x0, x1), slice(z0, z1)]
                hi = list(lo)
                hi[ax] = slice(lo[ax].start + 1, lo[ax].stop + 1)
                for fs in (tuple(lo), tuple(hi)):
                    assert bool((cd["alpha"][ax][fs] == 1).all() and (cd["beta"][ax][fs] == 0).all())
            # one more row or column on any side would leave the trivial set
            a = op.grid.n_abs
            assert (x0, x1, z0, z1) == (a[0], P[0] - a[0], a[1], P[1] - a[1])


def test_cfl_limit_and_ricker_wavelet():
    """tests/test_physics_wave.py:60-64 and :217-221: the leapfrog step limits of the order-2 and
    order-4 Laplacians, the refused safety factors, and the Ricker wavelet's peak, start and mean."""
    import math

    from nefi_b200.geometry import TimeAxis, ricker, stable_dt

    h = (0.1, 0.1)
    assert math.isclose(stable_dt(1.0, h, order=2, courant=1.0), 0.1 / math.sqrt(2))
    assert math.isclose(stable_dt(1.0, h, order=4, courant=1.0), 0.1 * math.sqrt(3 / 8))
    for bad in (0.0, 1.05):
        with pytest.raises(ConfigError):
            stable_dt(1.0, h, courant=bad)
    with pytest.raises(ConfigError):
        stable_dt(0.0, h)
    with pytest.raises(ConfigError):
        stable_dt(1.0, h, order=6)
    # the simulation step divides the observation step evenly and stays inside the limit
    ta = TimeAxis(100, 0.01, 2.5, h, 4, 0.9)
    assert ta.dt * ta.substeps == pytest.approx(0.01) and ta.dt <= stable_dt(2.5, h, 4, 0.9)
    assert ta.n_steps == 99 * ta.substeps
    t = torch.linspace(0, 1, 2001, dtype=torch.float64)
    w = ricker(t, 5.0)
    assert abs(float(w.max()) - 1.0) < 1e-6 and abs(float(t[w.argmax()]) - 1.2 / 5.0) < 1e-3
    assert abs(float(w[0])) < 1e-4 and abs(float(w.sum() * (t[1] - t[0]))) < 1e-4


def test_sensor_wrapped_3d_operator_shapes_and_resolution_cache():
    """tests/test_photoacoustic3d.py:27-37 with the drop-ins: a planar 8x8 sensor array on the top
    face, the trace shape independent of the grid, one cached operator per resolution, and the
    fidelity tag carried to the coarse operator."""
    from nefi_b200.misfit import SensorBandwidthB200

    dom = Domain((20, 20, 14), ((0.0, 3.0), (0.0, 3.0), (0.0, 2.1)))
    xs = (torch.arange(8, dtype=torch.float64) + 0.5) * 3.0 / 8
    X, Y = torch.meshgrid(xs, xs, indexing="ij")
    sensors = torch.stack([X.ravel(), Y.ravel(), torch.zeros(64, dtype=torch.float64)], -1)
    inner = WaveInitialConditionOperatorB200(dom, sensors, n_t=40, dt_obs=0.05, c=1.5, order=2,
                                             absorbing="sponge", absorb_width=0.45)
    op = SensorBandwidthB200(inner, 0.05, 2.0)
    assert op.homogeneity == 1.0 and op.primary == "p0" and op.required_fields() == ("p0",)
    assert op.output_shape((20, 20, 14)) == (64, 40) == op.output_shape((10, 10, 7))
    coarse = op.at_resolution((10, 10, 7))
    assert coarse is op.at_resolution((10, 10, 7)) and coarse.inner.domain.shape == (10, 10, 7)
    assert coarse.fidelity_tag == op.fidelity_tag and op.at_resolution((20, 20, 14)) is op
    assert SensorBandwidthB200(inner, 0.05, None).fidelity_tag == inner.fidelity_tag


def test_device_guard_follows_the_arguments(monkeypatch):
    """``_lib.on_device`` makes the arguments' GPU current for the library call: a CUDA tensor first,
    else a device name or an object's ``.device``; with no CUDA device in sight it only calls."""
    from nefi_b200 import _lib

    seen = []

    class Guard:
        def __init__(self, d):
            seen.append(torch.device(d))

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

    monkeypatch.setattr(torch.cuda, "device", Guard)

    class Holder:
        device = torch.device("cuda", 3)

    f = _lib.on_device(lambda *a, **k: "ran")
    assert f(1, torch.zeros(2), device="cpu") == "ran" and seen == []
    assert f(Holder()) == "ran" and seen == [torch.device("cuda", 3)]
    assert f([torch.zeros(1)], device="cuda:2") == "ran" and seen[-1] == torch.device("cuda", 2)
    assert f(torch.zeros(1), Holder(), device="cuda:1") == "ran" and seen[-1] == torch.device("cuda", 3)


def test_default_memory_budget_counts_the_allocators_idle_blocks(monkeypatch):
    dom = Domain((16, 16), ((0.0, 1.0), (0.0, 1.0)))
    op = WaveOperatorB200(dom, [[0.5, 0.5]], [[0.2, 0.2]], n_t=10, dt_obs=0.01, f0=5.0, c_max=2.5)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda d=None: (10 * 2**30, 180 * 2**30))
    monkeypatch.setattr(torch.cuda, "memory_reserved", lambda d=None: 50 * 2**30)
    monkeypatch.setattr(torch.cuda, "memory_allocated", lambda d=None: 20 * 2**30)
    assert op._budget(torch.device("cuda", 0)) == int(0.85 * 40 * 2**30)
    op2 = WaveOperatorB200(dom, [[0.5, 0.5]], [[0.2, 0.2]], n_t=10, dt_obs=0.01, f0=5.0, c_max=2.5,
                           memory_budget=123)
    assert op2._budget(torch.device("cuda", 0)) == 123


@pytest.mark.parametrize("seed", range(8))
def test_kernel_semantics_match_the_oracle_on_random_geometries(seed):
    """The kernels' semantics replayed in numpy over the real host tables (tests/kernel_model.py)
    against the float64 oracle on seeded random 2-D geometries: grid shape and spacing, layer kind
    and width, stencil order, substeps, several shots and receivers anywhere in the domain."""
    import random

    import oracle

    rnd = random.Random(seed)
    n0, n1 = rnd.randint(10, 28), rnd.randint(10, 28)
    h0, h1 = rnd.choice([0.04, 0.05]), rnd.choice([0.04, 0.05])
    ext = ((0.0, n0 * h0), (0.0, n1 * h1))
    absorbing = ["none", "sponge", "cerjan", "pml"][seed % 4]
    width = 0.0 if absorbing == "none" else rnd.choice([0.1, 0.2])
    lo = 0.5 * max(h0, h1) if absorbing == "none" else 0.0

    def point():
        return [rnd.uniform(lo, n0 * h0 - lo), rnd.uniform(lo, n1 * h1 - lo)]

    src = [point() for _ in range(rnd.randint(1, 3))]
    rec = [point() for _ in range(rnd.randint(1, 6))]
    dt_obs = rnd.choice([0.01, 0.02])  # long enough for the wave to cross the domain once
    n_t = int((n0 * h0 + n1 * h1) / 1.6 / dt_obs) + 10
    kw = dict(n_t=n_t, dt_obs=dt_obs, f0=rnd.choice([4.0, 6.0]), c_max=2.5,
              order=rnd.choice([2, 4]), absorbing=absorbing, absorb_width=width)
    g = np.random.default_rng(seed)
    c = np.clip(2.0 + 0.2 * g.standard_normal((n0, n1)), 1.6, 2.4)
    op = WaveOperatorB200(Domain((n0, n1), ext), src, rec, **kw)
    model = GhostModel(op._plan(CPU, torch.float64))
    C = model.medium(c, op.dt**2)
    gt = g.standard_normal((len(src), len(rec), kw["n_t"]))
    tr, gC, _, _ = model.run(C, op.n_steps, op.substeps, op.n_t, list(range(len(src))), grad_traces=gt)
    orc = oracle.OracleWave((n0, n1), ext, np.asarray(rec), sources=np.asarray(src), **kw)
    tr_o, gc_o = orc.fwi(c, gt, dtype=np.float64)
    assert np.linalg.norm(tr_o) > 0 and np.linalg.norm(gc_o) > 0  # the wave reaches the receivers
    assert rel_l2(tr, tr_o) < 1e-12, (absorbing, kw)
    assert rel_l2(model.fold_grad(c, op.dt**2, gC), gc_o) < 1e-11, (absorbing, kw)


@pytest.mark.parametrize("seed", range(4))
def test_kernel_semantics_match_the_oracle_on_random_3d_geometries(seed):
    """As above in 3-D (the plane-marching step's semantics): random box shapes, sponge, Cerjan or no
    layer, both orders, shots and receivers anywhere in the domain."""
    import random

    import oracle

    rnd = random.Random(100 + seed)
    n = [rnd.randint(6, 14) for _ in range(3)]
    h = 0.05
    ext = tuple((0.0, k * h) for k in n)
    absorbing = ["none", "sponge", "cerjan", "sponge"][seed]
    width = 0.0 if absorbing == "none" else 0.1
    lo = 0.5 * h if absorbing == "none" else 0.0

    def point():
        return [rnd.uniform(lo, k * h - lo) for k in n]

    src = [point() for _ in range(rnd.randint(1, 2))]
    rec = [point() for _ in range(rnd.randint(1, 5))]
    kw = dict(n_t=int(sum(n) * h / 1.6 / 0.01) + 5, dt_obs=0.01, f0=6.0, c_max=2.5,
              order=rnd.choice([2, 4]), absorbing=absorbing, absorb_width=width)
    g = np.random.default_rng(seed)
    c = np.clip(2.0 + 0.2 * g.standard_normal(n), 1.6, 2.4)
    gt = g.standard_normal((len(src), len(rec), kw["n_t"]))
    op = WaveOperatorB200(Domain(tuple(n), ext), src, rec, **kw)
    model = GhostModel(op._plan(CPU, torch.float64))
    C = model.medium(c, op.dt**2)
    tr, gC, _, _ = model.run(C, op.n_steps, op.substeps, op.n_t, list(range(len(src))), grad_traces=gt)
    orc = oracle.OracleWave(tuple(n), ext, np.asarray(rec), sources=np.asarray(src), **kw)
    tr_o, gc_o = orc.fwi(c, gt, dtype=np.float64)
    assert np.linalg.norm(tr_o) > 0
    assert rel_l2(tr, tr_o) < 1e-12, (absorbing, kw)
    assert rel_l2(model.fold_grad(c, op.dt**2, gC), gc_o) < 1e-11, (absorbing, kw)


@pytest.mark.parametrize("shape,extent", [((20, 31), ((0.0, 2.0), (-1.0, 2.1))),
                                          ((9, 12, 7), ((0.0, 0.9), (0.0, 1.2), (0.5, 1.2)))])
def test_padding_and_nearest_cells_match_the_oracle(shape, extent):
    """Replicate / zero padding and the cell containing a point (the receivers of time reversal)
    against the oracle's independent numpy versions, on points anywhere in the padded grid."""
    import oracle

    d = len(shape)
    rng = np.random.default_rng(2)
    op = WaveOperatorB200(Domain(shape, extent), [[e[0] + 0.3 * (e[1] - e[0]) for e in extent]],
                          [[e[0] + 0.6 * (e[1] - e[0]) for e in extent]], n_t=5, dt_obs=0.01, f0=5.0,
                          c_max=2.0, absorbing="sponge", absorb_width=0.25)
    orc = oracle.OracleWave(shape, extent, [[e[0] + 0.6 * (e[1] - e[0]) for e in extent]], n_t=5,
                            dt_obs=0.01, c_max=2.0, absorbing="sponge", absorb_width=0.25)
    x = rng.standard_normal((2, *shape))
    for mode in ("replicate", "zeros"):
        got = op.grid.pad(torch.tensor(x), mode).numpy()
        assert np.array_equal(got, orc.pad(x, mode))
    lo = [op.grid.lo_pad[ax] for ax in range(d)]
    span = [op.grid.padded_shape[ax] * op.grid.spacing[ax] for ax in range(d)]
    pts = np.stack([rng.uniform(lo[ax] - 0.1, lo[ax] + span[ax] + 0.1, 500) for ax in range(d)], 1)
    assert np.array_equal(op.grid.nearest_index(torch.tensor(pts)).numpy(), orc.nearest_cells(pts))



@pytest.mark.parametrize("edge", [False, True])
def test_pml_adjoint_tables_follow_the_interior_box(edge):
    """With a PML and a tiled interior box, the adjoint tile tables are built from the box's corner
    and hold the receiver-touched cells inside it (the box's adjoint launch adds their cotangents);
    the cells outside it (a receiver on the domain's face reaches the layer) are listed apart for the
    layer's launch."""
    shape, h = (60, 150), 0.01
    extent = ((0.0, shape[0] * h), (0.0, shape[1] * h))
    rec = [[0.02, 0.1 + 0.0123 * i] for i in range(100)]
    if edge:
        rec.append([0.0, 0.7])  # on the domain's face: the stencil's upper row lies in the layer
    op = WaveOperatorB200(Domain(shape, extent), [[0.05, 0.4]], rec, n_t=20, dt_obs=0.004, f0=25.0, c_max=2.5,
                          order=4, absorbing="pml", absorb_width=0.08)
    for dtype in (torch.float32, torch.float64):
        plan = op._plan(CPU, dtype)
        for tuning in [(0, 0, 0), (2, 2, 1, 2, 4, 2), (4, 2, 2, 4, 4, 1)]:
            if dtype == torch.float64 and 4 in tuning:
                continue
            plan.set_tuning(*tuning)
            assert plan.adj_tables_box == 1
            assert plan.layer_cell_index.numel() == (2 if edge else 0)
            a = plan.acquisition(1)
            assert a.adj_tables_box == 1 and tuple(a.adj_box_corner) == plan.adj_box_corner
            assert a.n_layer_cells == plan.layer_cell_index.numel()
            _check_tile_tables(plan)


def test_pml_layer_vectors_cover_the_layer_once_and_stay_in_bounds():
    """Replays the PML layer kernel's enumeration (pml2d.cuh: a thread per 16-byte vector of W cells,
    rows above the tiled box, the vectors left and right of it, rows below it) over random grids and
    boxes in the library's ghost layout: every layer cell is stored by exactly one lane, and every load
    and store offset of a vector (rows up to +-R, the neighbouring vectors of the centre row, faces
    P0 and P1) stays inside one field."""
    import ctypes as C
    import random

    from nefi_b200 import _lib

    lib = _lib.load()
    rnd = random.Random(7)
    for trial in range(400):
        r = rnd.choice([1, 2])
        W = rnd.choice([4, 2])  # float32, float64
        n0, n1 = rnd.randint(2 * r + 1, 70), rnd.randint(2 * r + 1, 110)
        g = _lib.Grid(ndim=2, order=2 * r, dtype=_lib.NW_F32 if W == 4 else _lib.NW_F64,
                      absorbing=_lib.NW_ABS_PML)
        g.n[0], g.n[1], g.n[2] = n0, n1, 1
        _lib.check(lib.nw_grid_layout(C.byref(g)))
        ld, origin, field = int(g.stride[0]), int(g.origin), int(g.field_elems)
        if trial % 4 == 0:
            kx0 = kx1 = kz0 = kz1 = 0
        else:  # a box as pml_tiled_box leaves it: first column rounded up to W, non-empty
            cx0 = rnd.randint(0, n0 - 1); cx1 = rnd.randint(cx0 + 1, n0)
            cz0 = rnd.randint(0, n1 - 1); cz1 = rnd.randint(cz0, n1)
            kz0 = -(-cz0 // W) * W
            kx0, kx1, kz1 = cx0, cx1, cz1
            if kz1 <= kz0:
                kx0 = kx1 = kz0 = kz1 = 0
        nvr = -(-n1 // W)
        vl, vr0 = kz0 // W, kz1 // W
        bw = vl + nvr - vr0
        top, mid = kx0 * nvr, (kx1 - kx0) * bw
        n_vec = top + mid + (n0 - kx1) * nvr
        seen = set()
        for t in range(n_vec):
            if t < top:
                x, m = divmod(t, nvr)
            elif t < top + mid:
                q, rr = divmod(t - top, bw)
                x, m = kx0 + q, (rr if rr < vl else vr0 + rr - vl)
            else:
                q, m = divmod(t - top - mid, nvr)
                x = kx1 + q
            zb = m * W
            i = origin + x * ld + zb
            assert i % W == 0 and ld % W == 0  # aligned 16-byte vectors
            mid_row = kx0 <= x < kx1
            for v in range(W):
                z = zb + v
                if z < n1 and (not mid_row or z < kz0 or z >= kz1):
                    assert (x, z) not in seen
                    seen.add((x, z))
            lo = min(i - W, i - r * ld, i - 1)
            hi = max(i + 2 * W - 1, i + r * ld + W - 1, i + ld + W - 1, i + W)
            assert 0 <= lo and hi < field, (n0, n1, r, W, x, zb)
        want = {(x, z) for x in range(n0) for z in range(n1) if not (kx0 <= x < kx1 and kz0 <= z < kz1)}
        assert seen == want, (n0, n1, kx0, kx1, kz0, kz1)
