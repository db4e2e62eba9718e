"""Pin the CPU oracle to the reference: its float64 results must reproduce the golden vectors the
reference produced (tests/golden/make_golden.py) to rounding, and its float32 results must stay
within single-precision distance of the reference's float32 results."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import cotangent, full_trace_shape, golden_names, load_golden, oracle_for, rel_l2

FWI = golden_names("fwi")
PAT = golden_names("pat")


def _fwi(case, dtype):
    orc = oracle_for(case)
    g = cotangent(full_trace_shape(case), case["seed"])
    tr, gc = orc.fwi(case["c"], g, dtype=dtype)
    return tr[:, :: case["rec_stride"]], gc


def _pat(case, dtype):
    orc = oracle_for(case)
    g = cotangent(full_trace_shape(case), case["seed"])
    return orc.pat(case["p0"], case["c"], g, dtype=dtype)


@pytest.mark.parametrize("name", FWI)
def test_oracle_fwi_float64_matches_reference(name):
    case = load_golden(name)
    tr, gc = _fwi(case, np.float64)
    assert rel_l2(tr, case["traces_f64"]) < 1e-12
    assert rel_l2(gc, case["grad_c_f64"]) < 1e-11


@pytest.mark.parametrize("name", PAT)
def test_oracle_pat_float64_matches_reference(name):
    case = load_golden(name)
    tr, gp, gc = _pat(case, np.float64)
    assert rel_l2(tr, case["traces_f64"]) < 1e-12
    assert rel_l2(gp, case["grad_p0_f64"]) < 1e-11
    assert rel_l2(gc, case["grad_c_f64"]) < 1e-11


@pytest.mark.parametrize("name", FWI)
def test_oracle_fwi_float32_close_to_reference_float32(name):
    case = load_golden(name)
    tr, gc = _fwi(case, np.float32)
    assert rel_l2(tr, case["traces_f32"]) < 1e-5
    assert rel_l2(gc, case["grad_c_f32"]) < 1e-4


@pytest.mark.parametrize("name", PAT)
def test_oracle_pat_float32_close_to_reference_float32(name):
    case = load_golden(name)
    tr, gp, gc = _pat(case, np.float32)
    assert rel_l2(tr, case["traces_f32"]) < 1e-5
    assert rel_l2(gp, case["grad_p0_f32"]) < 1e-4
    assert rel_l2(gc, case["grad_c_f32"]) < 1e-4


def test_oracle_detects_a_planted_error():
    """A perturbed oracle (sponge damping 5 % too strong) must fail the float64 pin."""
    case = load_golden("fwi_o4_sponge")
    orc = oracle_for(case)
    orc.B = 1.0 - (1.0 - orc.B) * 1.05
    g = cotangent(full_trace_shape(case), case["seed"])
    tr, gc = orc.fwi(case["c"], g)
    assert rel_l2(gc, case["grad_c_f64"]) > 1e-9


@pytest.mark.parametrize("name", golden_names("tr"))
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_oracle_time_reversal_matches_reference(name, dtype, tol):
    import oracle

    case = load_golden(name)
    kw = dict(case["kw"])
    orc = oracle.OracleWave(case["shape"], case["extent"], case["receivers"], n_t=case["traces"].shape[-1],
                            c_max=float(np.max(case["c"])), **kw)
    p0 = orc.time_reversal(case["traces"], case["c"], case["receivers"], dtype=dtype)
    ref = case["p0_f64"] if dtype == np.float64 else case["p0_f32"]
    assert rel_l2(p0, ref) < tol


@pytest.mark.parametrize("name", golden_names("gen"))
def test_oracle_supersampled_generation_matches_reference(name):
    """FP64 data generation on the refined grid (the operator's ``at_resolution``)."""
    import oracle

    case = load_golden(name)
    orc = oracle.OracleWave(case["fine"], case["extent"], case["receivers"], sources=case["sources"], **case["kw"])
    g = np.zeros(case["traces_f64"].shape)
    tr, _ = orc.fwi(case["c"], g, dtype=np.float64)
    assert rel_l2(tr, case["traces_f64"]) < 1e-12


@pytest.mark.parametrize("name", golden_names("misfit"))
def test_misfit_oracle_matches_reference(name):
    """The numpy misfit oracle against the reference's loss, gradient and filters (float64)."""
    import misfit_oracle as mo

    case = load_golden(name)
    kw = case["kw"]
    mask = case.get("mask")
    loss, grad = mo.band_limited_mse(case["pred"], case["obs"], kw["dt"], kw["f_max"], kw.get("taper", 0.3),
                                     kw["relative"], mask)
    assert abs(loss - float(case["loss_f64"])) <= 1e-12 * abs(float(case["loss_f64"]))
    assert rel_l2(grad, case["grad_f64"]) < 1e-12
    if kw["f_max"] is not None:
        assert rel_l2(mo.lowpass(case["pred"], kw["dt"], kw["f_max"], kw.get("taper", 0.3)), case["lowpass_f64"]) < 1e-13
    if case["sensor"] is not None:
        y, sl, sg = mo.sensor_mse(case["pred"], case["obs"], case["dt"], case["sensor"], mask)
        assert rel_l2(y, case["sensor_f64"]) < 1e-13
        assert abs(sl - float(case["sensor_loss_f64"])) <= 1e-12 * abs(float(case["sensor_loss_f64"]))
        assert rel_l2(sg, case["sensor_grad_f64"]) < 1e-12


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 1e-6)])
def test_oracle_pml_loops_match_the_array_restatement(dtype, tol):
    """The C loops of the PML run and its adjoint against the numpy array description of the same
    step, on a small seeded anisotropic grid with two shots."""
    import oracle

    rng = np.random.default_rng(5)
    shape, extent = (22, 30), ((0.0, 1.1), (0.0, 1.2))
    c = 2.0 + 0.3 * rng.random(shape)
    src, rec = [[0.3, 0.2], [0.7, 0.9]], [[0.9, y] for y in (0.1, 0.4, 0.8, 1.1)]
    orc = oracle.OracleWave(shape, extent, rec, sources=src, n_t=40, dt_obs=0.01, f0=5.0, c_max=2.4,
                            absorbing="pml", absorb_width=0.2)
    C2 = orc.c2dt2(c, dtype).reshape(-1)
    g = rng.standard_normal((2, len(rec), 40))
    a = orc._run_pml(C2, 2, None, None, g, dtype)
    b = orc._run_pml_numpy(C2, 2, None, None, g, dtype)
    for x, y in zip(a, b):
        assert rel_l2(x, y) < tol


def test_oracle_runs_in_shot_chunks_like_one_call():
    """Shot chunks (a history budget below one run's) give the results of one call."""
    case = load_golden("fwi_o4_pml")
    g = cotangent(full_trace_shape(case), case["seed"])
    one = oracle_for(case).fwi(case["c"], g)
    orc = oracle_for(case)
    orc.HISTORY_BYTES = 1
    chunked = orc.fwi(case["c"], g)
    assert np.array_equal(one[0], chunked[0]) and np.array_equal(one[1], chunked[1])


@pytest.mark.parametrize("seed", range(8))
def test_oracle_matches_reference_on_random_geometries(seed):
    """The float64 oracle against the reference's float64 runs of the seeded random geometries
    (tests/golden/random/random_<seed>.npz, stored in float32: agreement to that rounding), and the oracle's
    float32 arithmetic within twice the reference's own float32 error."""
    from pathlib import Path

    import oracle
    from random_geometry import random_geometry

    p = random_geometry(seed)
    ref = np.load(Path(__file__).parent / "golden" / "random" / f"random_{seed}.npz")
    orc = oracle.OracleWave(p["shape"], p["extent"], np.asarray(p["receivers"]), sources=np.asarray(p["sources"]),
                            **p["kw"])
    tr, gc = orc.fwi(p["c"], p["gt"], dtype=np.float64)
    assert rel_l2(tr, ref["traces_f64"]) < 1e-6 and rel_l2(gc, ref["grad_f64"]) < 1e-6
    tr32, gc32 = orc.fwi(p["c"], p["gt"], dtype=np.float32)
    r_tr = rel_l2(ref["traces_f32"], ref["traces_f64"])
    r_gc = rel_l2(ref["grad_f32"], ref["grad_f64"])
    assert rel_l2(tr32, ref["traces_f64"]) < max(1e-5, 2 * r_tr)
    assert rel_l2(gc32, ref["grad_f64"]) < max(1e-4, 2 * r_gc)
