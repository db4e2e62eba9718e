"""Python side of the CPU oracle: geometry in numpy float64 and the C time loop via ctypes.

TEST INFRASTRUCTURE ONLY (see wave_oracle.c). Used by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py; never by the ``nefi_b200`` product path.

This module restates the reference's grid conventions independently of ``nefi_b200.geometry``:
padded grid and layer depth (nefi/physics/wave.py:204-270), sponge and Cerjan coefficients
(nefi/physics/wave.py:431-475), CFL time axis (nefi/physics/timestep.py:177-207,
nefi/physics/wave.py:394-397), multilinear stencils and the source density
(nefi/physics/wave.py:272-318), the Ricker wavelet (nefi/physics/wave.py:101-111), replicate / zero
padding and its adjoint (nefi/physics/wave.py:222-246), the 2-D PML of ``_static`` and ``_step_fn``
(nefi/physics/wave.py:449-456, 476-501, 529-552; restated in numpy, with its adjoint derived by
hand: see ``_run_pml``), the photoacoustic start
``p^-1 = p0 + 1/2 c^2 dt^2 Lap p0`` (nefi/physics/wave.py:849-850) and the chain rule of
``c2dt2 = pad(c)^2 dt^2`` (nefi/physics/wave.py:718).
"""

from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class Geom(C.Structure):
    _fields_ = [("ndim", C.c_int), ("order", C.c_int), ("n", C.c_long * 3), ("w_center", C.c_double),
                ("w1", C.c_double * 3), ("w2", C.c_double * 3)]


def build(force: bool = False) -> Path:
    """Compile liboracle.so with gcc (``make -C oracle`` does the same)."""
    srcs = [HERE / "wave_oracle.c", HERE / "wave_oracle_impl.h"]
    if not force and LIB.exists() and all(s.stat().st_mtime <= LIB.stat().st_mtime for s in srcs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-o", str(tmp),
                    str(HERE / "wave_oracle.c")], check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        dp, lp = C.c_void_p, C.c_void_p
        for sfx in ("_f64", "_f32"):
            getattr(_lib, "oracle_laplacian" + sfx).argtypes = [C.POINTER(Geom), C.c_int, dp, dp]
            getattr(_lib, "oracle_forward" + sfx).argtypes = [
                C.POINTER(Geom), dp, dp, dp, C.c_int, C.c_int, lp, dp, C.c_int, dp, C.c_int, C.c_int,
                lp, dp, dp, dp, C.c_int, C.c_int, C.c_int, dp, dp]
            getattr(_lib, "oracle_adjoint" + sfx).argtypes = [
                C.POINTER(Geom), dp, dp, dp, C.c_int, C.c_int, C.c_int, lp, dp, dp, C.c_int, C.c_int,
                C.c_int, dp, dp, dp, dp]
            real = C.c_double if sfx == "_f64" else C.c_float
            getattr(_lib, "oracle_pml_forward" + sfx).argtypes = [
                C.POINTER(Geom), dp, dp, dp, dp, dp, dp, dp, dp, real, real, C.c_int, lp, dp, C.c_int, dp,
                C.c_int, C.c_int, lp, dp, dp, dp, C.c_int, C.c_int, C.c_int, dp, dp]
            getattr(_lib, "oracle_pml_adjoint" + sfx).argtypes = [
                C.POINTER(Geom), dp, dp, dp, dp, dp, dp, dp, dp, real, real, C.c_int, C.c_int, C.c_int, lp,
                dp, dp, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp]
    return _lib


def set_threads(n: int) -> None:
    """Thread count of the OpenMP loops (over shots)."""
    try:
        omp = C.CDLL("libgomp.so.1")
        omp.omp_set_num_threads(int(n))
    except OSError:
        pass


def _p(a):
    return None if a is None else a.ctypes.data


def ricker(t, f0, t0):
    a2 = (math.pi * f0 * (t - t0)) ** 2
    return (1.0 - 2.0 * a2) * np.exp(-a2)


class OracleWave:
    """CPU oracle of one wave operator (FWI when ``sources`` is given, else photoacoustic).

    Arguments mirror ``nefi.physics.wave.WaveOperator`` / ``WaveInitialConditionOperator``
    (nefi/physics/wave.py:610-632, 769-787), with the domain given as ``shape`` and ``extent``.
    """

    def __init__(self, shape, extent, receivers, *, n_t, dt_obs, c_max, order=4, absorbing="sponge",
                 absorb_width=None, absorb_R=1e-3, cerjan_gamma=0.3, courant=0.9, sources=None,
                 f0=None, t0=None, amplitude=1.0):
        if absorbing == "pml" and len(shape) != 2:
            raise ValueError("the PML is 1-D/2-D only (nefi/physics/wave.py:371-372)")
        self.shape = tuple(int(s) for s in shape)
        self.d = len(self.shape)
        self.extent = tuple((float(a), float(b)) for a, b in extent)
        self.h = tuple((hi - lo) / n for (lo, hi), n in zip(self.extent, self.shape))
        if absorb_width is None:
            absorb_width = 10.0 * max(self.h) if absorbing != "none" else 0.0
        W = float(absorb_width) if absorbing != "none" else 0.0
        self.a = tuple(int(math.ceil(W / h - 1e-9)) if W > 0 else 0 for h in self.h)
        self.P = tuple(n + 2 * a for n, a in zip(self.shape, self.a))
        self.lo = tuple(lo - a * h for (lo, _), a, h in zip(self.extent, self.a, self.h))
        self.order, self.absorbing = int(order), absorbing
        rho = {2: 4.0, 4: 16.0 / 3.0}[self.order]
        dt_max = courant * 2.0 / (c_max * math.sqrt(sum(rho / h**2 for h in self.h)))
        self.m = max(1, int(math.ceil(dt_obs / dt_max - 1e-12)))
        self.dt = dt_obs / self.m
        self.n_t = int(n_t)
        self.N = (self.n_t - 1) * self.m
        self.c_max, self.R, self.gamma = float(c_max), float(absorb_R), float(cerjan_gamma)
        self.rec_idx, self.rec_w = self._stencils(np.asarray(receivers, dtype=np.float64))
        self.sources = None if sources is None else np.asarray(sources, dtype=np.float64)
        if self.sources is not None:
            self.src_idx, sw = self._stencils(self.sources)
            self.src_w = sw / math.prod(self.h) * self.dt**2
            t = np.arange(self.N, dtype=np.float64) * self.dt
            t0 = 1.2 / f0 if t0 is None else t0
            self.wavelet = amplitude * ricker(t, f0, t0)
        self.geom = Geom()
        self.geom.ndim, self.geom.order = self.d, self.order
        for ax in range(3):
            self.geom.n[ax] = self.P[ax] if ax < self.d else 1
        co = {2: (-2.0, 1.0, 0.0), 4: (-2.5, 4.0 / 3.0, -1.0 / 12.0)}[self.order]
        wc = 0.0
        for ax in range(3):
            if ax < self.d:
                wc += co[0] / self.h[ax] ** 2
                self.geom.w1[ax] = co[1] / self.h[ax] ** 2
                self.geom.w2[ax] = co[2] / self.h[ax] ** 2
        self.geom.w_center = wc
        self._coefs()

    # -- geometry ----------------------------------------------------------------------------
    def _depth(self, ax):
        a, n = self.a[ax], self.shape[ax]
        pos = np.arange(n + 2 * a, dtype=np.float64) + 0.5
        if a == 0:
            return np.zeros_like(pos)
        return np.clip(np.maximum(a - pos, pos - (a + n)), 0.0, None) / a

    def _bcast(self, v, ax):
        s = [1] * self.d
        s[ax] = -1
        return v.reshape(s)

    def _face_depth(self, ax):
        a, n = self.a[ax], self.shape[ax]
        pos = np.arange(n + 2 * a + 1, dtype=np.float64)
        if a == 0:
            return np.zeros_like(pos)
        return np.clip(np.maximum(a - pos, pos - (a + n)), 0.0, None) / a

    def _coefs(self):
        self.A = self.B = None
        self.first_b_one = 0
        self.pml = None
        if not any(self.a) or self.absorbing == "none":
            return
        if self.absorbing == "pml":
            # zeta = 1.5 c_max ln(1/R) / (a h) xi^2 at cell centres and faces (wave.py:449-456, 476-501)
            zc, zf = [], []
            for ax, a in enumerate(self.a):
                zmax = 1.5 * self.c_max * math.log(1.0 / self.R) / (a * self.h[ax]) if a else 0.0
                zc.append(self._bcast(zmax * self._depth(ax) ** 2, ax))
                zf.append(self._bcast(zmax * self._face_depth(ax) ** 2, ax))
            zsum = np.broadcast_to(zc[0] + zc[1], self.P)
            dt = self.dt
            self.A = 1.0 / (1.0 + 0.5 * dt * zsum)
            self.B = 1.0 - 0.5 * dt * zsum
            pml = {"zz": np.broadcast_to(dt**2 * zc[0] * zc[1], self.P).copy(), "alpha": [], "beta": []}
            for ax in range(2):
                fshape = list(self.P)
                fshape[ax] += 1
                other = zc[1 - ax]
                den = 1.0 + 0.5 * dt * zf[ax]
                pml["alpha"].append(np.broadcast_to((1.0 - 0.5 * dt * zf[ax]) / den, fshape).copy())
                pml["beta"].append(np.broadcast_to(dt * (other - zf[ax]) / (den * self.h[ax]), fshape).copy())
            self.pml = pml
            return
        if self.absorbing == "sponge":
            sig = np.zeros(self.P)
            for ax, a in enumerate(self.a):
                if a:
                    smax = 3.0 * self.c_max * math.log(1.0 / self.R) / (a * self.h[ax])
                    sig = sig + smax * self._bcast(self._depth(ax), ax) ** 2
            half = 0.5 * sig * self.dt
            self.A, self.B = 1.0 / (1.0 + half), 1.0 - half
        else:
            xi = np.max(np.stack([np.broadcast_to(self._bcast(self._depth(ax), ax), self.P)
                                  for ax in range(self.d)]), axis=0)
            self.A = np.exp(-((self.gamma * xi) ** 2))
            self.B = self.A
            self.first_b_one = 1

    def _stencils(self, pts):
        idx_ax, w_ax = [], []
        for ax in range(self.d):
            h, lo, m = self.h[ax], self.lo[ax], self.P[ax]
            u = (pts[:, ax] - lo) / h - 0.5
            if (u < -1e-9).any() or (u > m - 1 + 1e-9).any():
                raise ValueError("point outside the simulation grid")
            u = np.clip(u, 0.0, m - 1)
            i0 = np.minimum(np.floor(u), max(m - 2, 0)).astype(np.int64)
            t = u - i0
            idx_ax.append(np.stack([i0, np.minimum(i0 + 1, m - 1)], 1))
            w_ax.append(np.stack([1.0 - t, t], 1))
        strides = [math.prod(self.P[ax + 1:]) for ax in range(self.d)]
        idx = np.zeros((pts.shape[0], 1), dtype=np.int64)
        w = np.ones((pts.shape[0], 1))
        for ax in range(self.d):
            idx = (idx[:, :, None] + strides[ax] * idx_ax[ax][:, None, :]).reshape(pts.shape[0], -1)
            w = (w[:, :, None] * w_ax[ax][:, None, :]).reshape(pts.shape[0], -1)
        return np.ascontiguousarray(idx), np.ascontiguousarray(w)

    def pad(self, x, mode):
        pw = [(0, 0)] * (x.ndim - self.d) + [(a, a) for a in self.a]
        return np.pad(x, pw, mode="edge" if mode == "replicate" else "constant")

    def crop(self, x):
        sl = (Ellipsis,) + tuple(slice(a, a + n) for a, n in zip(self.a, self.shape))
        return x[sl]

    def fold(self, g):
        """Adjoint of replicate padding: sums layer cells onto the edge cells they copy."""
        out = g
        for ax in range(self.d):
            a, n = self.a[ax], self.shape[ax]
            if a == 0:
                continue
            dim = out.ndim - self.d + ax
            core = np.take(out, np.arange(a, a + n), axis=dim).copy()
            lo = np.take(out, np.arange(0, a), axis=dim).sum(axis=dim)
            hi = np.take(out, np.arange(a + n, n + 2 * a), axis=dim).sum(axis=dim)
            idx0 = [slice(None)] * core.ndim
            idx0[dim] = 0
            idx1 = [slice(None)] * core.ndim
            idx1[dim] = n - 1
            core[tuple(idx0)] += lo
            core[tuple(idx1)] += hi
            out = core
        return out

    def laplacian(self, p, dtype=np.float64):
        p = np.ascontiguousarray(p, dtype=dtype)
        out = np.empty_like(p)
        nf = p.size // math.prod(self.P)
        fn = lib().oracle_laplacian_f64 if dtype == np.float64 else lib().oracle_laplacian_f32
        fn(C.byref(self.geom), nf, _p(p), _p(out))
        return out

    # -- runs --------------------------------------------------------------------------------
    # history bytes one call may hold; runs with more shots go through in chunks of shots (the shots
    # are independent, so the results are those of one call)
    HISTORY_BYTES = 2 << 30

    def _run(self, C2, n_shots, init_prev, init_cur, gtr, dtype, want_initial=False):
        per_shot = (self.N + 2) * math.prod(self.P) * np.dtype(dtype).itemsize
        chunk = max(1, int(self.HISTORY_BYTES // max(per_shot, 1)))
        if gtr is not None and n_shots > chunk:
            parts = []
            for s0 in range(0, n_shots, chunk):
                s1 = min(n_shots, s0 + chunk)
                sel = lambda a: None if a is None else np.asarray(a).reshape(n_shots, -1)[s0:s1]  # noqa: E731
                g = np.asarray(gtr).reshape(n_shots, -1, self.n_t)[s0:s1]
                parts.append(self._run_shots(C2, s1 - s0, sel(init_prev), sel(init_cur), g, dtype, want_initial, s0))
            cat = lambda i: None if parts[0][i] is None else np.concatenate([p[i] for p in parts], 0)  # noqa: E731
            return cat(0), cat(1), cat(2), cat(3)
        return self._run_shots(C2, n_shots, init_prev, init_cur, gtr, dtype, want_initial, 0)

    def _run_shots(self, C2, n_shots, init_prev, init_cur, gtr, dtype, want_initial, shot0):
        if self.pml is not None:
            return self._run_pml(C2, n_shots, init_prev, init_cur, gtr, dtype, shot0)
        L = lib()
        sfx = "_f64" if dtype == np.float64 else "_f32"
        cast = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dtype)  # noqa: E731
        C2, A, B = cast(C2), cast(self.A), cast(self.B)
        rec_w = cast(self.rec_w)
        src = self.sources is not None
        src_idx = np.ascontiguousarray(self.src_idx[shot0:shot0 + n_shots]) if src else None
        src_w = cast(self.src_w[shot0:shot0 + n_shots]) if src else None
        wav = cast(self.wavelet) if src else None
        cells = math.prod(self.P)
        traces = np.zeros((n_shots, self.rec_idx.shape[0], self.n_t), dtype=dtype)
        hist = np.zeros((self.N + 2, n_shots, cells), dtype=dtype) if gtr is not None else None
        ip, ic = cast(init_prev), cast(init_cur)
        getattr(L, "oracle_forward" + sfx)(
            C.byref(self.geom), _p(C2), _p(A), _p(B), self.first_b_one, n_shots, _p(src_idx), _p(src_w),
            src_idx.shape[1] if src else 0, _p(wav), self.rec_idx.shape[0], self.rec_idx.shape[1],
            _p(self.rec_idx), _p(rec_w), _p(ip), _p(ic), self.N, self.m, self.n_t, _p(traces), _p(hist))
        if gtr is None:
            return traces, None, None, None
        g = cast(gtr)
        gC = np.zeros((n_shots, cells), dtype=dtype)
        lam0 = np.zeros((n_shots, cells), dtype=dtype) if want_initial else None
        mu1 = np.zeros((n_shots, cells), dtype=dtype) if want_initial else None
        getattr(L, "oracle_adjoint" + sfx)(
            C.byref(self.geom), _p(C2), _p(A), _p(B), n_shots, self.rec_idx.shape[0],
            self.rec_idx.shape[1], _p(self.rec_idx), _p(rec_w), _p(hist), self.N, self.m, self.n_t,
            _p(g), _p(gC), _p(lam0), _p(mu1))
        return traces, gC, lam0, mu1

    def _run_pml(self, C2, S, init_prev, init_cur, gtr, dtype, shot0=0):
        """2-D PML run and, given cotangents, its exact adjoint, in C (``oracle_pml_forward`` /
        ``oracle_pml_adjoint``: the loops of ``_run_pml_numpy`` below, same operation order)."""
        L = lib()
        sfx = "_f64" if dtype == np.float64 else "_f32"
        cast = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dtype)  # noqa: E731
        C2, A, B, ZZ = cast(C2), cast(self.A), cast(self.B), cast(self.pml["zz"])
        al = [cast(x) for x in self.pml["alpha"]]
        be = [cast(x) for x in self.pml["beta"]]
        hx, hz = (0.5 / h for h in self.h)
        rec_w = cast(self.rec_w)
        src = self.sources is not None
        src_idx = np.ascontiguousarray(self.src_idx[shot0:shot0 + S]) if src else None
        src_w = cast(self.src_w[shot0:shot0 + S]) if src else None
        wav = cast(self.wavelet) if src else None
        cells = math.prod(self.P)
        n_rec, rec_pts = self.rec_idx.shape
        traces = np.zeros((S, n_rec, self.n_t), dtype=dtype)
        Lh = np.zeros((self.N, S, cells), dtype=dtype) if gtr is not None else None
        getattr(L, "oracle_pml_forward" + sfx)(
            C.byref(self.geom), _p(C2), _p(A), _p(B), _p(ZZ), _p(al[0]), _p(be[0]), _p(al[1]), _p(be[1]), hx, hz,
            S, _p(src_idx), _p(src_w), src_idx.shape[1] if src else 0, _p(wav), n_rec, rec_pts, _p(self.rec_idx),
            _p(rec_w), _p(cast(init_prev)), _p(cast(init_cur)), self.N, self.m, self.n_t, _p(traces), _p(Lh))
        if gtr is None:
            return traces, None, None, None
        g = cast(gtr)
        gC = np.zeros((S, cells), dtype=dtype)
        lam0 = np.zeros((S, cells), dtype=dtype)
        mu1 = np.zeros((S, cells), dtype=dtype)
        getattr(L, "oracle_pml_adjoint" + sfx)(
            C.byref(self.geom), _p(C2), _p(A), _p(B), _p(ZZ), _p(al[0]), _p(be[0]), _p(al[1]), _p(be[1]), hx, hz,
            S, n_rec, rec_pts, _p(self.rec_idx), _p(rec_w), _p(Lh), self.N, self.m, self.n_t, _p(g), _p(gC),
            _p(lam0), _p(mu1))
        return traces, gC, lam0, mu1

    def _run_pml_numpy(self, C2, S, init_prev, init_cur, gtr, dtype, shot0=0):
        """2-D PML run in numpy (all shots at once) and, given cotangents, its exact adjoint.

        Forward, step k (nefi/physics/wave.py:529-552), with face differences D+ (zero outside
        the grid, ``_face_diff``) and cell differences D- of face arrays:
            psi_k = alpha psi_{k-1} + beta D+ p^k                      (per axis, on faces)
            L_k   = Lap p^k + sum_ax (0.5/h) D-(psi_k + psi_{k-1})
            p^{k+1} = A (2 p^k - B p^{k-1} + C L_k - ZZ p^k + S w(k))
        Adjoint (derived by hand; D+^T = -D-, D-^T = -D+), with mu^k = A lambda^k:
            Psi_k  = alpha Psi_{k+1} - (0.5/h) D+(C mu^{k+1} + C mu^{k+2})
            lambda^k = R^T g_k + 2 mu^{k+1} - ZZ mu^{k+1} + Lap(C mu^{k+1})
                       - sum_ax D-(beta Psi_k) - B mu^{k+2}
            dJ/dC = sum_k mu^{k+1} L_k
        Returns (traces, per-shot dJ/dC, lambda^0, mu^1) like ``_run``.
        """
        P0, P1 = self.P
        cast = lambda a: np.asarray(a, dtype=dtype)  # noqa: E731
        Cf, A, B, ZZ = cast(C2).reshape(P0, P1), cast(self.A), cast(self.B), cast(self.pml["zz"])
        al = [cast(x) for x in self.pml["alpha"]]
        be = [cast(x) for x in self.pml["beta"]]
        half = [dtype(0.5 / h) for h in self.h]
        rec_idx, rec_w = self.rec_idx, cast(self.rec_w)
        src = self.sources is not None

        def lap(u):
            return self.laplacian(u.reshape(S, -1), dtype).reshape(S, P0, P1)

        def dplus(u, ax):  # cells -> faces, zero outside
            pw = [(0, 0), (0, 0), (0, 0)]
            pw[1 + ax] = (1, 1)
            return np.diff(np.pad(u, pw), axis=1 + ax)

        def dminus(f, ax):  # faces -> cells
            return np.diff(f, axis=1 + ax)

        pp = np.zeros((S, P0, P1), dtype) if init_prev is None else cast(init_prev).reshape(S, P0, P1).copy()
        pc = np.zeros((S, P0, P1), dtype) if init_cur is None else cast(init_cur).reshape(S, P0, P1).copy()
        psi = [np.zeros((S, P0 + 1, P1), dtype), np.zeros((S, P0, P1 + 1), dtype)]
        n_rec = rec_idx.shape[0]
        traces = np.zeros((S, n_rec, self.n_t), dtype)
        Ls = [] if gtr is not None else None
        for n in range(self.N + 1):
            if n % self.m == 0:
                flat = pc.reshape(S, -1)
                traces[:, :, n // self.m] = (flat[:, rec_idx] * rec_w).sum(-1)
            if n == self.N:
                break
            L = lap(pc)
            new = []
            for ax in range(2):
                ps = al[ax] * psi[ax] + be[ax] * dplus(pc, ax)
                L = L + dminus(ps + psi[ax], ax) * half[ax]
                new.append(ps)
            if Ls is not None:
                Ls.append(L)
            rhs = (dtype(2) * pc - B * pp) + Cf * L - ZZ * pc
            if src:
                flat = rhs.reshape(S, -1)
                for s in range(S):
                    np.add.at(flat[s], self.src_idx[shot0 + s], cast(self.src_w[shot0 + s]) * dtype(self.wavelet[n]))
            pp, pc, psi = pc, A * rhs, new
        if gtr is None:
            return traces, None, None, None
        g = cast(gtr)
        z = lambda: np.zeros((S, P0, P1), dtype)  # noqa: E731
        m1, m2 = z(), z()                          # mu^{k+1}, mu^{k+2}
        Psi = [np.zeros((S, P0 + 1, P1), dtype), np.zeros((S, P0, P1 + 1), dtype)]  # Psi_{k+1}
        gC = np.zeros((S, P0 * P1), dtype)
        lam0 = mu1 = None
        for k in range(self.N, -1, -1):
            lam = z()
            if k <= self.N - 1:
                q = Cf * m1
                s2 = q + Cf * m2
                Psi = [al[ax] * Psi[ax] - half[ax] * dplus(s2, ax) for ax in range(2)]
                lam = (dtype(2) * m1 - ZZ * m1) + lap(q)
                for ax in range(2):
                    lam = lam - dminus(be[ax] * Psi[ax], ax)
                lam = lam - B * m2
                gC += (m1 * Ls[k]).reshape(S, -1)
            if k % self.m == 0:
                flat = lam.reshape(S, -1)
                gv = g[:, :, k // self.m]
                for s in range(S):
                    np.add.at(flat[s], rec_idx.reshape(-1), (rec_w * gv[s][:, None]).reshape(-1))
            if k == 0:
                lam0, mu1 = lam.reshape(S, -1), m1.reshape(S, -1)
                break
            m2, m1 = m1, A * lam
        return traces, gC, lam0, mu1

    def nearest_cells(self, pts):
        """Flattened padded-grid index of the cell containing each point (nefi/physics/wave.py:302-310)."""
        pts = np.asarray(pts, dtype=np.float64)
        flat = np.zeros(pts.shape[0], dtype=np.int64)
        for ax in range(self.d):
            i = np.clip(np.floor((pts[:, ax] - self.lo[ax]) / self.h[ax]).astype(np.int64), 0, self.P[ax] - 1)
            flat = flat * self.P[ax] + i
        return flat

    def time_reversal(self, traces, c, receivers, dtype=np.float64):
        """Dirichlet time reversal (nefi/physics/wave.py:878-968): from rest, the receivers' cells are
        set to the traces at reversed time (linear in time between samples) after every step; the
        cropped field after the last step estimates p0. numpy, all in ``dtype``."""
        tr = np.asarray(traces, dtype=dtype)
        n_t = tr.shape[-1]
        m, N = self.m, self.N
        C2 = self.c2dt2_f64(c).astype(dtype).reshape(self.P)
        cells = self.nearest_cells(receivers)

        def rev(n):
            u = (n_t - 1) - n / m
            j0 = min(max(int(math.floor(u)), 0), n_t - 1)
            j1 = min(j0 + 1, n_t - 1)
            t = u - j0
            return dtype(1.0 - t) * tr[:, j0] + dtype(t) * tr[:, j1]

        pp = np.zeros(self.P, dtype)
        pc = np.zeros(self.P, dtype)
        pc.reshape(-1)[cells] = rev(0)
        A = None if self.A is None else np.asarray(self.A, dtype)
        B = None if self.B is None else np.asarray(self.B, dtype)
        psi = None
        if self.pml is not None:
            psi = [np.zeros((self.P[0] + 1, self.P[1]), dtype), np.zeros((self.P[0], self.P[1] + 1), dtype)]
        for n in range(N):
            L = self.laplacian(pc.reshape(1, -1), dtype).reshape(self.P)
            if psi is not None:
                new = []
                for ax in range(2):
                    pw = [(0, 0), (0, 0)]
                    pw[ax] = (1, 1)
                    ps = np.asarray(self.pml["alpha"][ax], dtype) * psi[ax] + \
                        np.asarray(self.pml["beta"][ax], dtype) * np.diff(np.pad(pc, pw), axis=ax)
                    L = L + np.diff(ps + psi[ax], axis=ax) * dtype(0.5 / self.h[ax])
                    new.append(ps)
                psi = new
                rhs = (dtype(2) * pc - B * pp) + C2 * L - np.asarray(self.pml["zz"], dtype) * pc
            else:
                b = 1 if B is None or (self.first_b_one and n == 0) else B
                rhs = (dtype(2) * pc - b * pp) + C2 * L
            nxt = rhs if A is None else A * rhs
            nxt.reshape(-1)[cells] = rev(n + 1)
            pp, pc = pc, nxt
        return self.crop(pc)

    def c2dt2_f64(self, c):
        """c^2 dt^2 of a fixed speed map, formed in float64 (nefi/physics/wave.py:814-820)."""
        cp = self.pad(np.broadcast_to(np.asarray(c, dtype=np.float64), self.shape), "replicate")
        return cp * cp * self.dt**2

    def c2dt2(self, c, dtype):
        cp = self.pad(np.asarray(c, dtype=dtype), "replicate")
        return (cp * cp) * dtype(self.dt**2)

    def fwi(self, c, grad_traces=None, dtype=np.float64):
        """Traces ``(n_src, n_rec, n_t)`` and, given cotangents, ``dJ/dc`` (float64)."""
        C2 = self.c2dt2(c, dtype).reshape(-1)
        S = self.sources.shape[0]
        tr, gC, _, _ = self._run(C2, S, None, None, grad_traces, dtype)
        if gC is None:
            return tr, None
        gsum = gC.astype(np.float64).sum(0).reshape(self.P)
        cp = self.pad(np.asarray(c, dtype=np.float64), "replicate")
        return tr, self.fold(2.0 * cp * self.dt**2 * gsum)

    def pat(self, p0, c, grad_traces=None, dtype=np.float64):
        """Photoacoustic traces ``(..., n_rec, n_t)``; given cotangents also ``dJ/dp0`` and
        ``dJ/dc`` (the latter through the c-dependence of every step and of ``p^-1``)."""
        p0 = np.asarray(p0, dtype=dtype)
        batch = p0.shape[: p0.ndim - self.d]
        S = int(math.prod(batch)) if batch else 1
        c = np.broadcast_to(np.asarray(c, dtype=dtype), self.shape)
        C2 = self.c2dt2(c, dtype).reshape(-1)
        p0p = self.pad(p0.reshape(S, *self.shape), "zeros").reshape(S, -1)
        lap0 = self.laplacian(p0p, dtype)
        pm1 = p0p + (dtype(0.5) * C2) * lap0
        g = None if grad_traces is None else np.asarray(grad_traces, dtype=dtype).reshape(S, -1, self.n_t)
        tr, gC, lam0, mu1 = self._run(C2, S, pm1, p0p, g, dtype, want_initial=True)
        tr = tr.reshape(*batch, -1, self.n_t)
        if gC is None:
            return tr, None, None
        lm1 = -(mu1 if self.B is None or self.first_b_one else self.B.reshape(-1).astype(dtype) * mu1)
        gp0p = (lam0 + lm1) + self.laplacian((dtype(0.5) * C2) * lm1, dtype)
        gp0 = self.crop(gp0p.reshape(S, *self.P)).reshape(*batch, *self.shape)
        gC = gC.astype(np.float64) + (0.5 * lm1.astype(np.float64)) * lap0.astype(np.float64)
        cp = self.pad(np.asarray(c, dtype=np.float64), "replicate")
        gc = self.fold(2.0 * cp * self.dt**2 * gC.sum(0).reshape(self.P))
        return tr, gp0, gc
