"""Shared test configuration: markers, golden-fixture loading and the CPU oracle."""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
for p in (str(ROOT), str(ROOT / "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)
# The NEFI package, when an installed copy is at hand (NEFI_REFERENCE, or the offline install under
# baseline/_ref): the B200 operators then subclass its Operator and raise its error types, and
# tests/test_gpu_dropin.py runs NEFI's own instances on them. Without it the package's mirror of
# the same API is used and those tests skip.
for p in (os.environ.get("NEFI_REFERENCE"), str(ROOT / "baseline" / "_ref")):
    if p and (Path(p) / "nefi" / "__init__.py").exists() and p not in sys.path:
        sys.path.append(p)
        break


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def golden_names(kind: str | None = None) -> list[str]:
    names = sorted(p.stem for p in GOLDEN.glob("*.npz"))
    if kind:
        names = [n for n in names if load_golden(n)["kind"] == kind]
    return names


_CACHE: dict = {}


def load_golden(name: str) -> dict:
    if name not in _CACHE:
        z = np.load(GOLDEN / f"{name}.npz")
        d = {k: z[k] for k in z.files if k != "meta"}
        d.update(json.loads(str(z["meta"])))
        d["name"] = name
        _CACHE[name] = d
    return _CACHE[name]


def cotangent(shape, seed) -> np.ndarray:
    """The seeded trace cotangent the golden generator used (tests/golden/make_golden.py)."""
    return torch.randn(tuple(shape), generator=torch.Generator().manual_seed(int(seed)),
                       dtype=torch.float64).numpy()


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_for(case: dict):
    import oracle

    kw = dict(case["kw"])
    if case["kind"] == "fwi":
        return oracle.OracleWave(case["shape"], case["extent"], case["receivers"], sources=case["sources"], **kw)
    kw.setdefault("c_max", float(np.max(case["c"])))  # the operator's default (nefi/physics/wave.py:793)
    return oracle.OracleWave(case["shape"], case["extent"], case["receivers"], **kw)


def full_trace_shape(case: dict) -> tuple[int, ...]:
    n_rec = case["receivers"].shape[0]
    if case["kind"] == "fwi":
        return (case["sources"].shape[0], n_rec, case["kw"]["n_t"])
    batch = case["p0"].shape[: case["p0"].ndim - len(case["shape"])]
    return (*batch, n_rec, case["kw"]["n_t"])


@pytest.fixture(scope="session")
def cuda_device():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
