"""Physics checks of the absorbing boundaries on the device, after the reference's own
tests/test_physics_wave.py:100-142: energy leaves the physical domain through every absorbing layer,
and the echo off a layer is small against a run in a domain large enough that no boundary is in reach.
"""

from __future__ import annotations

import pytest
import torch

from nefi_b200 import WaveOperatorB200
from nefi_b200._compat import Domain
from nefi_b200.geometry import stencil_weights

pytestmark = pytest.mark.gpu

F64 = torch.float64


def _shift(p, o, dim):
    out = torch.zeros_like(p)
    n = p.shape[dim]
    if o > 0:
        out.narrow(dim, o, n - o).copy_(p.narrow(dim, 0, n - o))
    else:
        out.narrow(dim, 0, n + o).copy_(p.narrow(dim, -o, n + o))
    return out


def _energy_fn(op, c):
    """Discrete leapfrog energy of the cropped state (nefi/physics/wave.py:171-189): the order-4
    Laplacian with zeros outside the physical domain, weighted by the cell volume."""
    wc, w1, w2 = stencil_weights(op.grid.spacing, 4)
    dv = op.grid.cell_volume

    def lap(p):
        out = wc * p
        for ax in (0, 1):
            for o, w in ((1, w1[ax]), (2, w2[ax])):
                out = out + w * (_shift(p, o, -2 + ax) + _shift(p, -o, -2 + ax))
        return out

    def energy(state, n):
        pp, p = (op.grid.crop(s) for s in state)
        kin = (p - pp) ** 2 / (c**2 * op.dt**2)
        return 0.5 * dv * (kin - p * lap(pp)).sum()

    return energy


@pytest.mark.parametrize("absorbing", ["pml", "sponge", "cerjan"])
def test_energy_decays_through_the_absorbing_layer(absorbing, cuda_device):
    """tests/test_physics_wave.py:119-124: with a 0.3-wide layer, less than 5 % of the peak energy
    is left in the physical domain at t = 1.49 s."""
    dom = Domain((40, 40), ((0.0, 1.0), (0.0, 1.0)))
    c = torch.full((40, 40), 1.0, dtype=F64)
    c[20:, :] = 1.5
    c = c.to(cuda_device)
    op = WaveOperatorB200(dom, [[0.5, 0.5]], [[0.2, 0.2]], n_t=150, dt_obs=0.01, f0=8.0, c_max=1.5,
                          order=4, absorbing=absorbing, absorb_width=0.3)
    rec = list(range(80, 1 + 149 * 2, 20))
    _, e = op.simulate(c, observe=_energy_fn(op, c), record=rec)
    e = torch.stack(e)
    assert float(e[-1] / e.max()) < 0.05, (absorbing, float(e[-1] / e.max()))


@pytest.mark.parametrize("absorbing,width,tol", [("pml", 0.2, 0.01), ("sponge", 0.6, 0.05),
                                                 ("cerjan", 0.6, 0.05)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_absorbing_boundary_reflection_is_small(absorbing, width, tol, dtype, cuda_device):
    """tests/test_physics_wave.py:127-142: the receiver sits 0.2 from the boundary; the largest
    difference against the same shot in a domain 9 times larger (no boundary in reach) stays below
    ``tol`` of the direct arrival."""
    c0, f0 = 2.0, 5.0
    small = Domain((60, 60), ((0.0, 1.2), (0.0, 1.2)))
    big = Domain((180, 180), ((-1.2, 2.4), (-1.2, 2.4)))
    kw = dict(n_t=220, dt_obs=0.004, f0=f0, c_max=c0)
    src, rec = [[0.6, 0.8]], [[0.6, 1.0]]
    ref = WaveOperatorB200(big, src, rec, absorbing="none", **kw)
    ref_tr = ref({"c": torch.full(big.shape, c0, dtype=dtype, device=cuda_device)})[0, 0].double()
    op = WaveOperatorB200(small, src, rec, absorbing=absorbing, absorb_width=width, **kw)
    tr = op({"c": torch.full(small.shape, c0, dtype=dtype, device=cuda_device)})[0, 0].double()
    refl = float((tr - ref_tr).abs().max() / ref_tr.abs().max())
    assert refl < tol, refl


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_steepest_descent_on_the_device_gradient_fits_the_data(dtype, cuda_device):
    """The end-to-end property of tests/test_instances_wave_family.py:58-65 (the inversion lowers the
    misfit and the anomaly error) with the device gradient driving a plain steepest descent with
    step halving: a 0.3 km/s Gaussian anomaly seen in transmission by 3 shots and 15 receivers.
    Six steps take the misfit below 5 % of its start and the model error below 80 % of its start
    (the reference's own gradient takes them to 1.2 % and 70 %)."""
    dom = Domain((48, 48), ((0.0, 0.96), (0.0, 0.96)))
    x = dom.physical_coords(dtype=F64)
    c_true = (2.0 + 0.3 * torch.exp(-((x - 0.48) ** 2).sum(-1) / (2 * 0.1**2))).to(cuda_device, dtype)
    src = [[0.1, y] for y in (0.2, 0.48, 0.76)]
    rec = [[0.86, 0.06 + 0.06 * i] for i in range(15)]
    op = WaveOperatorB200(dom, src, rec, n_t=150, dt_obs=0.004, f0=8.0, c_max=2.5, absorb_width=0.2)
    d = op({"c": c_true})
    c = torch.full((48, 48), 2.0, dtype=dtype, device=cuda_device)
    J0, g = op.misfit_gradient(c, d)
    J0, J = float(J0), float(J0)
    e0 = float((c - c_true).norm())
    alpha = 0.1
    for _ in range(6):
        for _ in range(5):
            cn = (c - alpha * (g / g.abs().max()).to(dtype)).clamp(1.5, 2.45)
            Jn, gn = op.misfit_gradient(cn, d)
            if float(Jn) < J:
                break
            alpha *= 0.5
        assert float(Jn) < J
        c, J, g = cn, float(Jn), gn
    assert J / J0 < 0.05, J / J0
    assert float((c - c_true).norm()) / e0 < 0.8
