"""CPU model of the fused misfit kernel's FFT (nefi_b200/csrc/misfit.cuh), no GPU needed: the same stage
groups, twiddle tables, decimation-in-frequency forward pass, bit-reversed response (written by the
library's host code) and decimation-in-time inverse pass, replayed in numpy, must reproduce the
oracle's low-pass and sensor filters (which reproduce the reference's) to float64 rounding."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from nefi_b200 import _lib


def make_groups(log2_len):
    sb, nb = [], []
    hi = log2_len
    while hi > 0:
        b = min(4, hi)
        sb.append(hi - b)
        nb.append(b)
        hi -= b
    off, tab_off = 16, []
    for t in range(log2_len):
        s = [sb[j] for j in range(len(sb)) if sb[j] <= t < sb[j] + nb[j]][0]
        tab_off.append(off)
        off += 1 << s
    return sb, nb, tab_off, off


def tables(log2_len, tab_off, tab_len):
    tab = np.zeros(tab_len, complex)
    for j in range(8):
        tab[j] = np.exp(-2j * np.pi * j / 16)
    for t in range(log2_len):
        n = (tab_off[t + 1] if t + 1 < log2_len else tab_len) - tab_off[t]
        tab[tab_off[t] + np.arange(n)] = np.exp(-1j * np.pi * np.arange(n) / (1 << t))
    return tab


def dif_group(v, low, sbit, nbits, tab, tab_off):
    for u in range(nbits - 1, -1, -1):
        half = 1 << u
        wl = tab[tab_off[sbit + u] + low]
        for k in range(1 << nbits):
            if k & half:
                continue
            a, b = v[k].copy(), v[k + half].copy()
            j = k & (half - 1)
            w = wl * (tab[j << (3 - u)] if j else 1)
            v[k], v[k + half] = a + b, (a - b) * w


def dit_group(v, low, sbit, nbits, tab, tab_off):
    for u in range(nbits):
        half = 1 << u
        wl = tab[tab_off[sbit + u] + low]
        for k in range(1 << nbits):
            if k & half:
                continue
            j = k & (half - 1)
            w = wl * (tab[j << (3 - u)] if j else 1)
            a, b = v[k].copy(), v[k + half] * np.conj(w)
            v[k], v[k + half] = a + b, a - b


def filt(x, hp, log2_len):
    """One filter as the kernel applies it: forward groups top-down, the lowest group with the
    response between its forward and inverse stages, inverse groups bottom-up."""
    L = 1 << log2_len
    sb, nb, tab_off, tab_len = make_groups(log2_len)
    tab = tables(log2_len, tab_off, tab_len)
    s = x.astype(complex).copy()

    def run(j, fn):
        gi = np.arange(L >> nb[j])
        low = gi & ((1 << sb[j]) - 1)
        base = ((gi >> sb[j]) << (sb[j] + nb[j])) | low
        idx = base[:, None] + (np.arange(1 << nb[j])[None, :] << sb[j])
        v = [s[idx[:, k]] for k in range(1 << nb[j])]
        fn(v, low, sb[j], nb[j], base)
        for k in range(1 << nb[j]):
            s[idx[:, k]] = v[k]

    G = len(sb)
    for j in range(G - 1):
        run(j, lambda v, low, sbit, n, base: dif_group(v, low, sbit, n, tab, tab_off))

    def middle(v, low, sbit, n, base):
        dif_group(v, low, sbit, n, tab, tab_off)
        for k in range(1 << n):
            v[k] = v[k] * hp[base + k]
        dit_group(v, low, sbit, n, tab, tab_off)

    run(G - 1, middle)
    for j in range(G - 2, -1, -1):
        run(j, lambda v, low, sbit, n, base: dit_group(v, low, sbit, n, tab, tab_off))
    return s


@pytest.mark.parametrize("n_t,dt,f,taper", [(30, 0.01, 20.0, 0.3), (101, 0.004, 40.0, 0.5), (257, 0.002, 100.0, 0.0)])
def test_kernel_fft_decomposition_reproduces_the_filters(n_t, dt, f, taper):
    import misfit_oracle as mo

    lib = _lib.load()
    k = lib.nw_filter_log2_len(n_t)
    L = 1 << k
    rng = np.random.default_rng(n_t)
    xa, xb = rng.standard_normal((2, n_t))
    z = np.zeros(L, complex)
    z[:n_t] = xa + 1j * xb  # two traces as one complex sequence, as a CTA holds them
    for kind, ref in ((_lib.NW_FILTER_LOWPASS, lambda x: mo.lowpass(x, dt, f, taper)),
                      (_lib.NW_FILTER_GAUSSIAN, lambda x: mo.gaussian_lowpass(x, dt, f))):
        hp = np.zeros(L)
        _lib.check(lib.nw_filter_response(kind, n_t, C.c_double(dt), C.c_double(f), C.c_double(taper), 1,
                                          hp.ctypes.data))
        out = filt(z, hp, k)[:n_t]
        want = ref(np.stack([xa, xb]))
        scale = np.abs(want).max()
        assert np.abs(out.real - want[0]).max() <= 1e-13 * scale
        assert np.abs(out.imag - want[1]).max() <= 1e-13 * scale
