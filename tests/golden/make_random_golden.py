"""Run the reference NEFI package on the seeded random geometries of tests/random_geometry.py and
store its float32 and float64 results: traces of ``op({"c": c})`` and the gradient of
``sum(traces * gt)`` taken with ``torch.autograd`` through the reference's unrolled loop
(grad_mode "autograd"). Written as float32 (the comparisons they serve are at the 1e-5 level) to
tests/golden/random/random_<seed>.npz.

    python tests/golden/make_random_golden.py /path/to/reference
    NEFI_REFERENCE=/path/to/reference python tests/golden/make_random_golden.py -
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
_arg = sys.argv[1] if len(sys.argv) > 1 else "-"
if _arg == "-" and not os.environ.get("NEFI_REFERENCE"):
    sys.exit("usage: make_random_golden.py /path/to/reference (or '-' with NEFI_REFERENCE set)")
REF = Path(os.environ["NEFI_REFERENCE"] if _arg == "-" else _arg)
sys.path.insert(0, str(REF))
sys.path.insert(0, str(HERE.parent))

from nefi.domain import Domain  # noqa: E402
from nefi.physics.wave import WaveOperator  # noqa: E402
from random_geometry import SEEDS, random_geometry  # noqa: E402


def run(p: dict, dtype: torch.dtype):
    op = WaveOperator(Domain(p["shape"], p["extent"]), p["sources"], p["receivers"], grad_mode="autograd", **p["kw"])
    c = torch.tensor(p["c"], dtype=dtype, requires_grad=True)
    tr = op({"c": c})
    (gc,) = torch.autograd.grad((tr * torch.tensor(p["gt"], dtype=dtype)).sum(), c)
    return tr.detach().numpy().astype(np.float32), gc.numpy().astype(np.float32)


def main() -> None:
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    (HERE / "random").mkdir(exist_ok=True)
    for seed in SEEDS:
        p = random_geometry(seed)
        tr64, gc64 = run(p, torch.float64)
        tr32, gc32 = run(p, torch.float32)
        np.savez_compressed(HERE / "random" / f"random_{seed}.npz", traces_f64=tr64, grad_f64=gc64, traces_f32=tr32,
                            grad_f32=gc32)
        e_tr = np.linalg.norm(tr32.astype(np.float64) - tr64) / np.linalg.norm(tr64)
        e_gc = np.linalg.norm(gc32.astype(np.float64) - gc64) / np.linalg.norm(gc64)
        print(f"seed {seed} {p['kw']['absorbing']} {p['shape']} n_t {p['kw']['n_t']}: reference float32 vs "
              f"float64 traces {e_tr:.2e}, gradient {e_gc:.2e}", flush=True)


if __name__ == "__main__":
    main()
