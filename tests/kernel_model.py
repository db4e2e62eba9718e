"""A numpy model of the CUDA kernels' semantics over the ghost layout (test helper).

It consumes the very host tables the operators hand to the library (``DevicePlan`` built on the
CPU: ghost offsets, stencil corners and weights, the adjoint receiver table, absorbing
coefficients) and replays the drivers' loop structure (nefi_b200/csrc/wave_capi.cu), so the host
logic can be checked against the oracle without a GPU.
"""

from __future__ import annotations

import itertools
import math

import numpy as np


class GhostModel:
    def __init__(self, plan):
        g = plan.g
        self.plan, self.g = plan, g
        self.d = g.ndim
        self.P = tuple(g.n[ax] for ax in range(self.d))
        self.s = [int(g.stride[ax]) for ax in range(self.d)]
        self.r = int(g.radius)
        grids = np.meshgrid(*[np.arange(n) for n in self.P], indexing="ij")
        self.I = g.origin + sum(grids[ax].astype(np.int64) * self.s[ax] for ax in range(self.d))
        self.I = self.I.reshape(-1)
        self.coords = [gr.reshape(-1) for gr in grids]
        lo = [g.core_lo[ax] for ax in range(self.d)]
        hi = [g.core_hi[ax] for ax in range(self.d)]
        self.layer = np.zeros(self.I.shape, dtype=bool)
        for ax in range(self.d):
            self.layer |= (self.coords[ax] < lo[ax]) | (self.coords[ax] >= hi[ax])
        self.A = None if plan.A is None else plan.A.numpy().astype(np.float64)
        self.B = None if plan.B is None else plan.B.numpy().astype(np.float64)
        self.w1 = [g.w1[ax] for ax in range(self.d)]
        self.w2 = [g.w2[ax] for ax in range(self.d)]
        self.wc = g.w_center
        self.F = int(g.field_elems)
        self.pml = None
        if plan.pml is not None:
            self.pml = {"ZZ": plan.pml["ZZ"].numpy().astype(np.float64),
                        "alpha": [a.numpy().astype(np.float64) for a in plan.pml["alpha"]],
                        "beta": [b.numpy().astype(np.float64) for b in plan.pml["beta"]],
                        "h2": list(plan.pml["half_inv_h"])}

    def lap(self, p):
        I = self.I
        out = self.wc * p[I]
        for ax in range(self.d):
            s = self.s[ax]
            out = out + self.w1[ax] * (p[I - s] + p[I + s])
            if self.r == 2:
                out = out + self.w2[ax] * (p[I - 2 * s] + p[I + 2 * s])
        return out

    def medium(self, c, dt2):
        C = np.zeros(self.F)
        n_abs = [self.plan.n_abs[ax] for ax in range(self.d)]
        phys = [np.clip(self.coords[ax] - n_abs[ax], 0, c.shape[ax] - 1) for ax in range(self.d)]
        C[self.I] = c[tuple(phys)] ** 2 * dt2
        return C

    def step(self, C, prev, cur, n, shot, b_one):
        pl = self.plan
        rhs_b = np.ones(self.I.shape)
        if self.B is not None and not b_one:
            rhs_b = np.where(self.layer, self.B[self.I], 1.0)
        rhs = (2.0 * cur[self.I] - rhs_b * prev[self.I]) + C[self.I] * self.lap(cur)
        nxt = np.zeros(self.F)
        nxt[self.I] = rhs
        if pl.has_source:
            corner = pl.src_corner[shot].numpy()
            w = pl.src_weight[shot].numpy().astype(np.float64)
            wn = float(pl.wavelet[n])
            for k, bits in enumerate(itertools.product((0, 1), repeat=self.d)):
                off = self.g.origin + sum((corner[ax] + bits[ax]) * self.s[ax] for ax in range(self.d))
                nxt[off] += w[k] * wn
        if self.A is not None:
            nxt[self.I] = np.where(self.layer, self.A[self.I] * nxt[self.I], nxt[self.I])
        return nxt

    def sample(self, p):
        idx = self.plan.rec_index.numpy()
        w = self.plan.rec_weight.numpy().astype(np.float64)
        return (w * p[idx]).sum(-1)

    def inject(self, mu, g_j, apply_a):
        pl = self.plan
        cells = pl.cell_index.numpy()
        ptr = pl.cell_ptr.numpy()
        rec = pl.cell_rec.numpy()
        w = pl.cell_weight.numpy().astype(np.float64)
        for c in range(len(cells)):
            acc = sum(w[e] * g_j[rec[e]] for e in range(ptr[c], ptr[c + 1]))
            a = self.A[cells[c]] if (apply_a and self.A is not None) else 1.0
            mu[cells[c]] += a * acc

    def _pml_faces(self, u, fo, ax, adjoint, other=None):
        """The kernel's face pair (f = x, x+1) of axis ``ax`` for every interior cell."""
        I, s, pm = self.I, self.s[ax], self.pml
        al, be = pm["alpha"][ax], pm["beta"][ax]
        if not adjoint:
            f0 = be[I] * (u[I] - u[I - s]) + al[I] * fo[I]
            f1 = be[I + s] * (u[I + s] - u[I]) + al[I + s] * fo[I + s]
        else:
            sm, s0, sp = u[I - s] + other[I - s], u[I] + other[I], u[I + s] + other[I + s]
            f0 = al[I] * fo[I] - pm["h2"][ax] * (s0 - sm)
            f1 = al[I + s] * fo[I + s] - pm["h2"][ax] * (sp - s0)
        last = self.coords[ax] == self.P[ax] - 1
        new = np.zeros(self.F)
        new[I] = f0
        new[I[last] + s] = f1[last]
        return f0, f1, new

    def run_pml(self, C, n_steps, m, n_t, shots, init=None, grad_traces=None):
        """``run`` for the 2-D PML (pml2d_step): face fields stored at the cell index of the face."""
        I, pm = self.I, self.pml
        S = len(shots)
        traces = np.zeros((S, self.plan.n_rec, n_t))
        Ls = []
        for si, shot in enumerate(shots):
            prev = np.zeros(self.F) if init is None else init[0][si].copy()
            cur = np.zeros(self.F) if init is None else init[1][si].copy()
            psi = [np.zeros(self.F), np.zeros(self.F)]
            L_s = []
            for n in range(n_steps):
                if n % m == 0:
                    traces[si, :, n // m] = self.sample(cur)
                L = self.lap(cur)
                new = []
                for ax in range(2):
                    f0, f1, nf = self._pml_faces(cur, psi[ax], ax, False)
                    L = L + pm["h2"][ax] * ((f1 + psi[ax][I + self.s[ax]]) - (f0 + psi[ax][I]))
                    new.append(nf)
                L_s.append(L)
                rhs = (2.0 * cur[I] - self.B[I] * prev[I]) + C[I] * L - pm["ZZ"][I] * cur[I]
                nxt = np.zeros(self.F)
                nxt[I] = rhs
                if self.plan.has_source:
                    corner = self.plan.src_corner[shot].numpy()
                    w = self.plan.src_weight[shot].numpy().astype(np.float64)
                    for k, bits in enumerate(itertools.product((0, 1), repeat=2)):
                        off = self.g.origin + sum((corner[ax] + bits[ax]) * self.s[ax] for ax in range(2))
                        nxt[off] += w[k] * float(self.plan.wavelet[n])
                nxt[I] = self.A[I] * nxt[I]
                prev, cur, psi = cur, nxt, new
            traces[si, :, n_steps // m] = self.sample(cur)
            Ls.append(L_s)
        if grad_traces is None:
            return traces, None, None, None
        gC = np.zeros((S, self.F))
        lam0 = np.zeros((S, self.F))
        mu1_out = np.zeros((S, self.F))
        for si in range(S):
            q1, q2 = np.zeros(self.F), np.zeros(self.F)  # C mu^{n+1}, C mu^{n+2}
            Psi = [np.zeros(self.F), np.zeros(self.F)]
            qs = {}
            for n in range(n_steps, -1, -1):
                lapq = self.lap(q1)
                term = np.zeros(I.shape)
                new = []
                for ax in range(2):
                    f0, f1, nf = self._pml_faces(q1, Psi[ax], ax, True, other=q2)
                    be = pm["beta"][ax]
                    term = term + (be[I + self.s[ax]] * f1 - be[I] * f0)
                    new.append(nf)
                Psi = new
                o = (2.0 * q1[I] - pm["ZZ"][I] * q1[I]) + C[I] * (lapq - term) - self.B[I] * q2[I]
                out = np.zeros(self.F)
                out[I] = self.A[I] * o if n >= 1 else o
                if n % m == 0:  # C R^T g_n, scaled by A like the rest of the step
                    inj = np.zeros(self.F)
                    self.inject(inj, grad_traces[si, :, n // m], False)
                    out[I] += (self.A[I] if n >= 1 else 1.0) * C[I] * inj[I]
                if n <= n_steps - 1:
                    gC[si, I] += q1[I] * Ls[si][n]
                qs[n] = out
                q1, q2 = out, q1
            with np.errstate(divide="ignore", invalid="ignore"):
                lam0[si, I] = qs[0][I] / C[I]
                mu1_out[si, I] = (qs[1][I] / C[I]) if n_steps >= 1 else 0.0
            gC[si, I] = gC[si, I] / C[I]  # C dJ/dC -> dJ/dC
        return traces, gC, lam0, mu1_out

    def run(self, C, n_steps, m, n_t, shots, init=None, grad_traces=None):
        """Forward (and adjoint) for every shot; returns traces, per-shot dJ/dC, lambda0, mu1."""
        if self.pml is not None:
            return self.run_pml(C, n_steps, m, n_t, shots, init, grad_traces)
        S = len(shots)
        n_rec = self.plan.n_rec
        traces = np.zeros((S, n_rec, n_t))
        hist = []
        for si, shot in enumerate(shots):
            prev = np.zeros(self.F) if init is None else init[0][si].copy()
            cur = np.zeros(self.F) if init is None else init[1][si].copy()
            h = [prev, cur]
            for n in range(n_steps):
                if n % m == 0:
                    traces[si, :, n // m] = self.sample(cur)
                nxt = self.step(C, prev, cur, n, shot, n == 0 and self.plan.first_b_one)
                prev, cur = cur, nxt
                h.append(cur)
            traces[si, :, n_steps // m] = self.sample(cur)
            hist.append(h)
        if grad_traces is None:
            return traces, None, None, None
        gC = np.zeros((S, self.F))
        lam0 = np.zeros((S, self.F))
        mu1_out = np.zeros((S, self.F))
        for si in range(S):
            mu = {n_steps + 1: np.zeros(self.F), n_steps + 2: np.zeros(self.F)}
            for n in range(n_steps, -1, -1):
                m1, m2 = mu[n + 1], mu[n + 2]
                out = np.zeros(self.F)
                q = C * m1
                lam = (2.0 * m1[self.I] + self.lap(q))
                b = np.where(self.layer, self.B[self.I], 1.0) if self.B is not None else 1.0
                lam = lam - b * m2[self.I]
                if n >= 1 and self.A is not None:
                    lam = np.where(self.layer, self.A[self.I] * lam, lam)
                out[self.I] = lam
                if n % m == 0:
                    self.inject(out, grad_traces[si, :, n // m], n >= 1)
                if n <= n_steps - 1:
                    gC[si, self.I] += m1[self.I] * self.lap(hist[si][n + 1])
                mu[n] = out
            lam0[si] = mu[0]
            mu1_out[si] = mu[1]
        return traces, gC, lam0, mu1_out

    def fold_grad(self, c, dt2, gC):
        """Float64 reduction over shots and the replicate-padding adjoint (reduce_grad_kernel)."""
        n_abs = [self.plan.n_abs[ax] for ax in range(self.d)]
        tot = gC.sum(0)[self.I].reshape(self.P)
        out = np.zeros(c.shape)
        for idx in itertools.product(*[range(k) for k in c.shape]):
            sl = []
            for ax, i in enumerate(idx):
                a, mph = n_abs[ax], c.shape[ax]
                lo = 0 if i == 0 else i + a
                hi = mph + 2 * a - 1 if i == mph - 1 else i + a
                sl.append(slice(lo, hi + 1))
            out[idx] = 2.0 * c[idx] * dt2 * tot[tuple(sl)].sum()
        return out

    def dense(self, flat):
        return flat[..., self.I].reshape(*flat.shape[:-1], *self.P)


def product(xs):
    return math.prod(xs)
