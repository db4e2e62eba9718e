"""The device's delta16 snapshot encoder against the CPU model of the codec (test_snapshot_codec.py),
bitwise: a checkpointed forward run stores exact snapshots in one pool and delta16 snapshots in
another; every block of the delta16 pool (codes, step, anchor) must be the model's encoding of the
same block of the exact pool (p^{n0} and the level difference p^{n0} - p^{n0-1}, and with a PML the
two face fields). The decoder is covered by the gradient tests that run through it (its grid-cell
mask by the bitwise depth-1 / depth-2 comparisons)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden
from test_gpu_parity import make_op
from test_snapshot_codec import encode

pytestmark = pytest.mark.gpu


def _pool(op, x, key):
    tr = op({key: x})
    fn = tr.grad_fn
    while not hasattr(fn, "run"):  # views between the output and the autograd function
        fn = fn.next_functions[0][0]
    run = fn.run
    torch.cuda.synchronize()
    return run, run.snap.cpu().numpy()


@pytest.mark.parametrize("name,dtype,every", [("fwi_o4_sponge", torch.float32, 10),
                                              ("fwi_o4_pml", torch.float32, 10),
                                              ("fwi_o4_sponge", torch.float64, 7),
                                              ("pat3d_o2_sponge", torch.float32, 10)])
def test_delta16_pool_is_the_model_encoding_of_the_exact_snapshots(name, dtype, every, cuda_device):
    case = load_golden(name)
    key = "c" if case["kind"] == "fwi" else "p0"
    x = torch.tensor(case[key], dtype=dtype, device=cuda_device, requires_grad=True)  # storage is kept for a gradient
    run_e, exact = _pool(make_op(case, grad_mode="checkpoint", checkpoint_every=every, snapshot="exact"), x, key)
    run_d, d16 = _pool(make_op(case, grad_mode="checkpoint", checkpoint_every=every, snapshot="delta16"), x, key)
    plan = run_e.plan
    S, field = run_e.n_shots, plan.field
    assert field % 32 == 0
    slots = 4 if plan.pml is not None else 2
    nblk = field // 32
    esz = torch.finfo(dtype).bits // 8
    fdt = np.float32 if dtype == torch.float32 else np.float64
    per_exact = slots * S * field * esz
    vals_b = slots * S * nblk * 64
    scale_b = slots * S * nblk * 4
    per_d16 = (vals_b + 2 * scale_b + 255) // 256 * 256
    n_snap = exact.size // per_exact
    assert n_snap >= 2 and d16.size >= n_snap * per_d16
    for j in range(n_snap):
        lv = exact[j * per_exact:(j + 1) * per_exact].view(fdt).reshape(slots, S, field)
        # slot inputs as the encoder forms them: in the computation's dtype, then rounded to float32
        inputs = [lv[1], lv[1] - lv[0]] + ([lv[2], lv[3]] if slots == 4 else [])
        blk = np.stack(inputs).astype(np.float32).reshape(-1, 32)
        codes, step, anchor, _ = encode(blk)
        assert np.abs(codes).max() <= 32767
        base = j * per_d16
        got_codes = d16[base:base + vals_b].view(np.int16).reshape(-1, 32)
        got_step = d16[base + vals_b:base + vals_b + scale_b].view(np.float32)
        got_anchor = d16[base + vals_b + scale_b:base + vals_b + 2 * scale_b].view(np.float32)
        np.testing.assert_array_equal(got_codes, codes.astype(np.int16), err_msg=f"codes of snapshot {j}")
        np.testing.assert_array_equal(got_step.view(np.uint32), step[:, 0].view(np.uint32),
                                      err_msg=f"steps of snapshot {j}")
        np.testing.assert_array_equal(got_anchor.view(np.uint32), anchor[:, 0].view(np.uint32),
                                      err_msg=f"anchors of snapshot {j}")
