"""Seeded random 2-D FWI geometries: grid shape and spacing, every layer kind, order, several shots,
receivers anywhere in the domain, long enough for the wave to cross the domain. Shared by the device
parity test (tests/test_gpu_parity.py) and the script that runs the reference on them
(tests/golden/make_random_golden.py), so both see the same problems."""

from __future__ import annotations

import random

import numpy as np


def random_geometry(seed: int) -> dict:
    """The problem of `seed`: shape, extent, sources, receivers, operator keyword arguments, the
    sound speed c and the trace cotangent gt (float64 numpy arrays)."""
    rnd = random.Random(seed)
    n0, n1 = rnd.randint(10, 90), rnd.randint(10, 170)
    h0, h1 = rnd.choice([0.04, 0.05]), rnd.choice([0.04, 0.05])
    ext = ((0.0, n0 * h0), (0.0, n1 * h1))
    absorbing = ["none", "sponge", "cerjan", "pml"][seed % 4]
    width = 0.0 if absorbing == "none" else rnd.choice([0.1, 0.2])
    lo = 0.5 * max(h0, h1) if absorbing == "none" else 0.0

    def point():
        return [rnd.uniform(lo, n0 * h0 - lo), rnd.uniform(lo, n1 * h1 - lo)]

    src = [point() for _ in range(rnd.randint(1, 5))]
    rec = [point() for _ in range(rnd.randint(1, 12))]
    dt_obs = rnd.choice([0.01, 0.02])  # long enough for the wave to cross the domain once
    n_t = int((n0 * h0 + n1 * h1) / 1.6 / dt_obs) + 10
    kw = dict(n_t=n_t, dt_obs=dt_obs, f0=rnd.choice([4.0, 6.0]), c_max=2.5,
              order=rnd.choice([2, 4]), absorbing=absorbing, absorb_width=width)
    g = np.random.default_rng(seed)
    c = np.clip(2.0 + 0.2 * g.standard_normal((n0, n1)), 1.6, 2.4)
    gt = g.standard_normal((len(src), len(rec), kw["n_t"]))
    return {"shape": (n0, n1), "extent": ext, "sources": src, "receivers": rec, "kw": kw, "c": c, "gt": gt}


SEEDS = range(8)
