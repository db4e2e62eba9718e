"""The C-ABI library loads, exports every function include/nefi_wave.h declares, and its host-only
entry points (layout, sizes, errors) behave; no CUDA device is needed."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from nefi_b200 import _lib
from nefi_b200.build import build

HEADER = Path(__file__).resolve().parents[1] / "include" / "nefi_wave.h"


def declared_functions(header: Path = HEADER) -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(nw_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build()
    return _lib.load()


def test_every_declared_symbol_is_exported_and_bound(lib):
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_lib.EXPORTED) == names


def test_abi_version_and_arch(lib):
    assert lib.nw_abi_version() == _lib.ABI_VERSION == 6
    assert lib.nw_built_arch() == 1000


@pytest.mark.parametrize("ndim,order", [(2, 2), (2, 4), (3, 2), (3, 4)])
def test_ghost_layout_keeps_every_stencil_read_in_bounds(lib, ndim, order):
    g = _lib.Grid()
    g.ndim, g.order, g.dtype = ndim, order, _lib.NW_F32
    n = (13, 7, 37)[:ndim]
    for ax in range(3):
        g.n[ax] = n[ax] if ax < ndim else 1
    _lib.check(lib.nw_grid_layout(C.byref(g)))
    r = order // 2
    assert g.radius == r
    ld = g.stride[ndim - 2]  # row pitch of the contiguous axis
    assert ld % 32 == 0 and ld >= n[-1] + r
    # the lowest and highest neighbour reads (one axis at a time) stay inside [0, field_elems)
    reach = max(r * g.stride[ax] for ax in range(ndim))
    last = [k - 1 for k in n]
    hi_cell = g.origin + sum(last[ax] * g.stride[ax] for ax in range(ndim))
    assert g.origin - reach >= 0 and hi_cell + reach < g.field_elems
    # a neighbour outside the grid along one axis never aliases an interior cell
    interior = set()
    import itertools

    for idx in itertools.product(*[range(k) for k in n]):
        interior.add(g.origin + sum(i * g.stride[ax] for ax, i in enumerate(idx)))
    for idx in itertools.product(*[range(k) for k in n]):
        base = g.origin + sum(i * g.stride[ax] for ax, i in enumerate(idx))
        for ax in range(ndim):
            for o in range(1, r + 1):
                for sgn in (-1, 1):
                    j = idx[ax] + sgn * o
                    if not 0 <= j < n[ax]:
                        assert base + sgn * o * g.stride[ax] not in interior


def test_invalid_arguments_report_errors(lib):
    g = _lib.Grid()
    g.ndim, g.order = 1, 2
    rc = lib.nw_grid_layout(C.byref(g))
    assert rc == _lib.NW_ERR_UNSUPPORTED
    assert b"ndim" in lib.nw_last_error()
    g.ndim, g.order = 2, 6
    assert lib.nw_grid_layout(C.byref(g)) == _lib.NW_ERR_ARG
    with pytest.raises(_lib.LibraryError, match="order"):
        _lib.check(lib.nw_grid_layout(C.byref(g)))


def test_snapshot_pool_sizes(lib):
    g = _lib.Grid()
    g.ndim, g.order, g.dtype = 2, 4, _lib.NW_F32
    g.n[0], g.n[1], g.n[2] = 552, 552, 1
    _lib.check(lib.nw_grid_layout(C.byref(g)))
    exact = lib.nw_snapshot_bytes(C.byref(g), 16, 10, _lib.NW_SNAP_EXACT)
    assert exact == 10 * 2 * 16 * g.field_elems * 4
    for kind in (_lib.NW_SNAP_F16, _lib.NW_SNAP_BF16, _lib.NW_SNAP_I16):
        half = lib.nw_snapshot_bytes(C.byref(g), 16, 10, kind)
        # 2 bytes per element plus one float scale per 32-element block
        assert 0.53 * exact < half < 0.54 * exact


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(_lib.LibraryError, match="missing"):
        _lib.load(tmp_path / "libnefiwave.so")


def test_filter_length_and_response_limits(lib):
    assert lib.nw_filter_log2_len(0) == _lib.NW_ERR_ARG
    assert [lib.nw_filter_log2_len(n) for n in (1, 32, 33, 4096, 4097, 8192)] == [6, 6, 7, 13, 14, 14]
    out = np.empty(1 << 15, dtype=np.float64)
    for kind in (_lib.NW_FILTER_LOWPASS, _lib.NW_FILTER_GAUSSIAN):
        assert lib.nw_filter_response(kind, 8193, 1e-3, 50.0, 0.3, _lib.NW_F64, out.ctypes.data) == \
            _lib.NW_ERR_UNSUPPORTED
        assert lib.nw_filter_response(kind, 8192, 1e-3, 50.0, 0.3, _lib.NW_F64, out.ctypes.data) == _lib.NW_OK
        assert lib.nw_filter_response(kind, 100, 0.0, 50.0, 0.3, _lib.NW_F64, out.ctypes.data) == _lib.NW_ERR_ARG
    assert lib.nw_filter_response(7, 100, 1e-3, 50.0, 0.3, _lib.NW_F64, out.ctypes.data) == _lib.NW_ERR_ARG
    assert lib.nw_filter_response(_lib.NW_FILTER_LOWPASS, 100, 1e-3, 50.0, 1.5, _lib.NW_F64,
                                  out.ctypes.data) == _lib.NW_ERR_ARG


def test_grid_validation_runs_before_any_device_call(lib):
    """Entry points refuse a bad grid on the host: NULL, a 3-D PML, an unknown dtype, a padded extent
    below 2, a field of 2^31 elements or more."""
    shape = (C.c_int32 * 4)()
    assert lib.nw_forward(None, None, None, None, None, None, 0, 0, None, None) == _lib.NW_ERR_ARG
    assert b"NULL" in lib.nw_last_error()

    def grid(**kw):
        g = _lib.Grid()
        g.ndim, g.order, g.dtype, g.absorbing = 2, 4, _lib.NW_F32, _lib.NW_ABS_SPONGE
        g.n[0], g.n[1], g.n[2] = 64, 64, 1
        for k, v in kw.items():
            if k == "n":
                g.n[0], g.n[1], g.n[2] = v
            else:
                setattr(g, k, v)
        assert lib.nw_grid_layout(C.byref(g)) == _lib.NW_OK
        return g

    t = _lib.Tuning()
    assert lib.nw_tile_shape(C.byref(grid()), C.byref(t), shape) == _lib.NW_OK
    cases = [(dict(ndim=3, n=(16, 16, 16), absorbing=_lib.NW_ABS_PML), _lib.NW_ERR_UNSUPPORTED),
             (dict(dtype=9), _lib.NW_ERR_ARG),
             (dict(n=(1, 64, 1)), _lib.NW_ERR_ARG),
             (dict(n=(50000, 50000, 1)), _lib.NW_ERR_ARG)]
    for kw, rc in cases:
        assert lib.nw_tile_shape(C.byref(grid(**kw)), C.byref(t), shape) == rc, kw


def test_misaligned_device_buffers_are_refused_on_the_host(lib):
    """Fields move in 16-byte vectors: a medium or storage buffer off a 16-byte boundary is refused
    before any launch (the addresses below are never dereferenced)."""
    g = _lib.Grid()
    g.ndim, g.order, g.dtype, g.absorbing = 2, 4, _lib.NW_F32, _lib.NW_ABS_SPONGE
    g.n[0], g.n[1], g.n[2] = 64, 64, 1
    assert lib.nw_grid_layout(C.byref(g)) == _lib.NW_OK
    a = _lib.Acquisition()
    a.n_shots = 1
    t = _lib.Time()
    t.substeps, t.n_t, t.n_steps = 1, 2, 1
    for bad in ("c2dt2", "coef_a", "ring", "segbuf", "snap"):
        m = _lib.Medium()
        m.c2dt2, m.coef_a, m.coef_b = 0x10000, 0x20000, 0x30000
        st = _lib.Storage()
        st.ring = 0x40000
        target = m if bad in ("c2dt2", "coef_a") else st
        setattr(target, bad, 0x50004)
        rc = lib.nw_forward(C.byref(g), C.byref(m), C.byref(a), C.byref(t), C.byref(st), None, 0, 1, None, None)
        assert rc == _lib.NW_ERR_ARG, bad
        assert b"16-byte" in lib.nw_last_error(), bad


def test_binding_structs_match_the_header_layout(tmp_path):
    """Every descriptor struct of the ctypes binding has the C header's size and field offsets, as a C
    compiler lays them out (a binding whose fields drift from the header passes garbage silently)."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    pairs = {"nw_grid": _lib.Grid, "nw_tuning": _lib.Tuning, "nw_acquisition": _lib.Acquisition,
             "nw_medium": _lib.Medium, "nw_time": _lib.Time, "nw_storage": _lib.Storage,
             "nw_batch_problem": _lib.BatchProblem, "nw_traces": _lib.Traces}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "nefi_wave.h"', "int main(void) {"]
    for cname, cls in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    include = Path(__file__).resolve().parents[1] / "include"
    subprocess.run([cc, "-std=c99", f"-I{include}", str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, key, value = line.split()
        got[(cname, key)] = int(value)
    for cname, cls in pairs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
