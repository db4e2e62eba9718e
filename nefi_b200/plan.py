"""Device-side tables of one operator at one (device, dtype): the ``nw_*`` descriptors.

A :class:`DevicePlan` owns the constant device tensors (absorbing coefficients in the ghost layout,
source/receiver stencils, the adjoint receiver table, the wavelet) and the ctypes descriptors that
point at them. It is built once per operator, device and dtype and reused by every call, so a
forward or adjoint sweep does no host-side geometry work.
"""

from __future__ import annotations

import ctypes as C
import functools
import math

import torch

from . import _lib
from ._compat import ConfigError
from .geometry import PaddedGrid, cerjan_taper, pml_coefficients, sponge_coefficients, stencil_weights


def ghost_layout(grid_struct: _lib.Grid) -> _lib.Grid:
    _lib.check(_lib.load().nw_grid_layout(C.byref(grid_struct)))
    return grid_struct


def make_grid(grid: PaddedGrid, order: int, dtype: torch.dtype, absorbing: str) -> _lib.Grid:
    g = _lib.Grid()
    g.ndim = grid.d
    g.order = order
    g.dtype = _lib.dtype_code(dtype)
    g.absorbing = {"none": _lib.NW_ABS_NONE, "sponge": _lib.NW_ABS_SPONGE, "cerjan": _lib.NW_ABS_CERJAN,
                   "pml": _lib.NW_ABS_PML}[absorbing if any(grid.n_abs) else "none"]
    for ax in range(3):
        if ax < grid.d:
            g.n[ax] = grid.padded_shape[ax]
            g.core_lo[ax] = grid.n_abs[ax]
            g.core_hi[ax] = grid.n_abs[ax] + grid.shape[ax]
        else:
            g.n[ax], g.core_lo[ax], g.core_hi[ax] = 1, 0, 1
    wc, w1, w2 = stencil_weights(grid.spacing, order)
    g.w_center = wc
    for ax in range(3):
        g.w1[ax] = w1[ax] if ax < grid.d else 0.0
        g.w2[ax] = w2[ax] if ax < grid.d else 0.0
    return ghost_layout(g)


def to_ghost(g: _lib.Grid, dense: torch.Tensor, fill: float = 0.0) -> torch.Tensor:
    """Place a padded-grid array ``(*P)`` into a flat ghost-layout buffer (host or device)."""
    out = torch.full((g.field_elems,), fill, dtype=dense.dtype, device=dense.device)
    view = ghost_view(g, out)
    view.copy_(dense)
    return out


def ghost_view(g: _lib.Grid, flat: torch.Tensor) -> torch.Tensor:
    """Strided view ``(..., *P)`` of the interior cells of ghost-layout field(s) in ``flat``."""
    lead = flat.shape[:-1]
    r = g.radius
    body = flat[..., g.guard:]
    if g.ndim == 2:
        rows = body.shape[-1] // g.stride[0]
        v = body.view(*lead, rows, g.stride[0])
        return v[..., r:r + g.n[0], : g.n[1]]
    planes = body.shape[-1] // g.stride[0]
    v = body.view(*lead, planes, g.stride[0] // g.stride[1], g.stride[1])
    return v[..., r:r + g.n[0], : g.n[1], : g.n[2]]


def to_ghost_faces(g: _lib.Grid, faces: torch.Tensor, ax: int) -> torch.Tensor:
    """Place a 2-D face array (padded shape with ``P_ax + 1`` along ``ax``) into a ghost-layout field:
    face ``f`` at the cell index ``f``, so face ``P_ax`` lands in the first ghost row / column."""
    out = torch.zeros((g.field_elems,), dtype=faces.dtype)
    body = out[g.guard:].view(-1, g.stride[0])
    r = g.radius
    body[r:r + faces.shape[0], : faces.shape[1]].copy_(faces)
    return out


def ghost_offsets(g: _lib.Grid, corner: torch.Tensor) -> torch.Tensor:
    """Ghost-layout offsets ``(n, 2^d)`` of the stencil corners (same ordering as the weights)."""
    d = g.ndim
    out = torch.full((corner.shape[0], 1), int(g.origin), dtype=torch.long)
    for ax in range(d):
        hi = (corner[:, ax] + 1).clamp(max=g.n[ax] - 1)
        pair = torch.stack([corner[:, ax], hi], 1) * int(g.stride[ax])
        out = (out[:, :, None] + pair[:, None, :]).flatten(1)
    return out


def pml_core_box(co: dict) -> tuple[int, int, int, int]:
    """The box ``(x0, x1, z0, z1)`` of padded cells where the PML step reduces exactly to the plain
    leapfrog update (``A = B = 1``, ``ZZ = 0``, and on both faces of both axes ``alpha = 1``,
    ``beta = 0``, in the computation's dtype), so the step may skip the face fields there; the
    faces of such cells never leave zero in the forward, and their cotangents meet a zero ``beta``.
    ``(0, 0, 0, 0)`` when no such box exists."""
    A, B, ZZ = co["A"], co["B"], co["ZZ"]
    ok = (A == 1) & (B == 1) & (ZZ == 0)
    for ax in range(2):
        face = (co["alpha"][ax] == 1) & (co["beta"][ax] == 0)  # P_ax + 1 faces along ax
        lo = face.narrow(ax, 0, face.shape[ax] - 1)
        hi = face.narrow(ax, 1, face.shape[ax] - 1)
        ok &= (lo & hi).expand(ok.shape)
    if not bool(ok.any()):
        return (0, 0, 0, 0)
    rows = torch.nonzero(ok.any(dim=1)).flatten()
    cols = torch.nonzero(ok.any(dim=0)).flatten()
    x0, x1, z0, z1 = int(rows[0]), int(rows[-1]) + 1, int(cols[0]), int(cols[-1]) + 1
    if not bool(ok[x0:x1, z0:z1].all()):
        return (0, 0, 0, 0)
    return (x0, x1, z0, z1)


class DevicePlan:
    """Constant device tables of one operator (``op``) for ``device`` and ``dtype``."""

    def __init__(self, op, device: torch.device, dtype: torch.dtype) -> None:
        self.device, self.dtype = device, dtype
        grid: PaddedGrid = op.grid
        self.pgrid = grid
        self.g = make_grid(grid, op.order, dtype, op.absorbing)
        self.n_abs = (C.c_int32 * 3)(*(list(grid.n_abs) + [0] * (3 - grid.d)))
        self.field = int(self.g.field_elems)
        cast = {"device": device, "dtype": dtype}
        # absorbing coefficients (interior cells are exactly 1, ghost cells 0)
        self.A = self.B = None
        if self.g.absorbing == _lib.NW_ABS_SPONGE:
            a, b = sponge_coefficients(grid, op.c_max, op.absorb_R, op.dt)
            self.A = to_ghost(self.g, a.to(dtype)).to(device)
            self.B = to_ghost(self.g, b.to(dtype)).to(device)
        elif self.g.absorbing == _lib.NW_ABS_CERJAN:
            tp = cerjan_taper(grid, op.cerjan_gamma)
            self.A = to_ghost(self.g, tp.to(dtype)).to(device)
            self.B = self.A
        self.pml = None
        if self.g.absorbing == _lib.NW_ABS_PML:
            co = pml_coefficients(grid, op.c_max, op.absorb_R, op.dt)
            self.A = to_ghost(self.g, co["A"].to(dtype)).to(device)
            self.B = to_ghost(self.g, co["B"].to(dtype)).to(device)
            self.pml = {"ZZ": to_ghost(self.g, co["ZZ"].to(dtype)).to(device),
                        "alpha": [to_ghost_faces(self.g, co["alpha"][ax].to(dtype), ax).to(device) for ax in range(2)],
                        "beta": [to_ghost_faces(self.g, co["beta"][ax].to(dtype), ax).to(device) for ax in range(2)],
                        "half_inv_h": [0.5 / h for h in grid.spacing],
                        "core": pml_core_box({k: (v.to(dtype) if torch.is_tensor(v) else [t.to(dtype) for t in v])
                                              for k, v in co.items()})}
        self.first_b_one = 1 if self.g.absorbing == _lib.NW_ABS_CERJAN else 0
        # receivers
        corner, w = grid.point_stencils(op.receivers)
        self.n_rec = int(corner.shape[0])
        idx = ghost_offsets(self.g, corner)
        self.rec_index = idx.to(device)
        self.rec_weight = w.to(**cast)
        # adjoint table: cells touched by receiver stencils, entries in (receiver, corner) order
        flat = idx.reshape(-1)
        rec_of = torch.arange(self.n_rec).repeat_interleave(idx.shape[1])
        order = torch.argsort(flat, stable=True)
        cells, counts = torch.unique_consecutive(flat[order], return_counts=True)
        self.n_cells = int(cells.numel())
        self.cell_index = cells.to(device)
        ptr = torch.zeros(self.n_cells + 1, dtype=torch.int32)
        ptr[1:] = torch.cumsum(counts, 0).to(torch.int32)
        self.cell_ptr = ptr.to(device)
        self.cell_rec = rec_of[order].to(torch.int32).to(device)
        self.cell_weight = w.reshape(-1)[order].to(**cast)
        # sources (FWI only)
        self.has_source = hasattr(op, "sources")
        if self.has_source:
            sc, sw = grid.point_stencils(op.sources)
            self.src_corner = sc.to(torch.int32).to(device)
            self.src_weight = (sw / grid.cell_volume * op.dt**2).to(**cast)
            self.wavelet = op.wavelet().to(**cast)
        self.time = _lib.Time(op.n_steps, op.substeps, op.n_t, self.first_b_one)
        self._corner = corner
        self._cells = cells
        self.set_tuning(*(getattr(op, "tuning", None) or ()))

    def set_tuning(self, vz: int = 0, rx: int = 0, shots_per_cta: int = 0, adj_vz: int = 0, adj_rx: int = 0,
                   adj_shots_per_cta: int = 0, depth: int = 0) -> None:
        """Choose the 2-D launch shapes (0 = library default) and the forward steps per launch
        (``depth`` 2: two, on 2-D grids without a PML), and build the per-tile tables."""
        t = _lib.Tuning(int(vz), int(rx), int(shots_per_cta), int(adj_vz), int(adj_rx), int(adj_shots_per_cta),
                        int(depth))
        shape = (C.c_int32 * 4)()
        _lib.check(_lib.load().nw_tile_shape(C.byref(self.g), C.byref(t), shape))
        self.tuning = t
        # forward steps per launch as the library resolved them (two need a ring of four levels)
        self.ring_levels = 4 if (int(depth) == 2 and self.g.ndim == 2 and self.pml is None) else 3
        self.tile = (shape[0], shape[1])       # forward steps
        self.adj_tile = (shape[2], shape[3])   # adjoint steps
        self.tiles_z = self.adj_tiles_z = 0
        self.rec_corner = self.tile_rec_ptr = self.tile_rec_list = None
        self.tile_cell_ptr = self.tile_cell_local = self.tile_cell_gid = None
        self.adj_tables_box, self.adj_box_corner = 0, (0, 0)
        self.layer_cell_index = self.layer_cell_gid = None
        if self.g.ndim == 2:
            self._build_tile_tables()

    def _build_tile_tables(self) -> None:
        """Per-tile receiver tables (forward tile shape) and adjoint-source tables (adjoint tile
        shape) for the 2-D step kernels.

        A receiver belongs to the tile holding its stencil's lower corner (its other corners lie
        in that tile's one-cell halo); a receiver-touched cell belongs to the tile containing it.
        Lists keep ascending receiver / cell order inside each tile.
        """
        g = self.g
        TX, TZ = self.tile
        tiles_z = -(-g.n[1] // TZ)
        n_tiles = tiles_z * -(-g.n[0] // TX)
        corner = self._corner
        tile_of = (corner[:, 0] // TX) * tiles_z + corner[:, 1] // TZ
        order = torch.argsort(tile_of, stable=True)
        rptr = torch.zeros(n_tiles + 1, dtype=torch.int64)
        rptr[1:] = torch.cumsum(torch.bincount(tile_of, minlength=n_tiles), 0)
        AX, AZ = self.adj_tile
        rel = self._cells - int(g.origin)
        x, z = rel // int(g.stride[0]), rel % int(g.stride[0])
        # the adjoint tile grid: from cell (0, 0) over the whole grid, or, with a PML and a tiled
        # interior box, from the box's corner over the box, holding the touched cells inside it, the
        # others listed apart (the box's adjoint launch and the layer's then add the cotangents)
        ox, oz, ex, ez = 0, 0, int(g.n[0]), int(g.n[1])
        gid_all = torch.arange(self.n_cells)
        box = self.pml_tiled_box(AX, AZ)
        if box is not None and self.n_cells > 0:
            bx0, bx1, bz0, bz1 = box
            inside = (x >= bx0) & (x < bx1) & (z >= bz0) & (z < bz1)
            ox, oz, ex, ez = bx0, bz0, bx1, bz1
            self.adj_tables_box, self.adj_box_corner = 1, (bx0, bz0)
            self.layer_cell_index = self._cells[~inside].to(torch.int32).to(self.device)
            self.layer_cell_gid = gid_all[~inside].to(torch.int32).to(self.device)
            x, z, gid_all = x[inside], z[inside], gid_all[inside]
        x, z = x - ox, z - oz
        adj_tiles_z = -(-(ez - oz) // AZ)
        n_adj_tiles = adj_tiles_z * -(-(ex - ox) // AX)
        ctile = (x // AX) * adj_tiles_z + z // AZ
        corder = torch.argsort(ctile, stable=True)
        cptr = torch.zeros(n_adj_tiles + 1, dtype=torch.int64)
        cptr[1:] = torch.cumsum(torch.bincount(ctile, minlength=n_adj_tiles), 0)
        local = (x % AX) * AZ + z % AZ
        dev, i32 = self.device, torch.int32
        self.tiles_z, self.adj_tiles_z = tiles_z, adj_tiles_z
        self.rec_corner = corner.to(i32).contiguous().to(dev)
        self.tile_rec_ptr = rptr.to(i32).to(dev)
        self.tile_rec_list = order.to(i32).to(dev)
        self.tile_cell_ptr = cptr.to(i32).to(dev)
        self.tile_cell_local = local[corder].to(i32).to(dev)
        self.tile_cell_gid = gid_all[corder].to(i32).to(dev)

    def pml_tiled_box(self, tx: int, tz: int):
        """The PML's interior box that the tiled kernels of a (tx, tz) tile step, as the library derives
        it (wave_capi.cu ``pml_tiled_box``): the core box with its first column rounded up to a
        16-byte chunk, or None when there is no PML or the box is smaller than one tile."""
        if self.pml is None:
            return None
        x0, x1, z0, z1 = (int(v) for v in self.pml["core"])
        epc = 16 // (torch.finfo(self.dtype).bits // 8)
        z0 = -(-z0 // epc) * epc
        if x1 - x0 < tx or z1 - z0 < tz:
            return None
        return x0, x1, z0, z1

    def n_acc(self, n_shots: int) -> int:
        """Gradient accumulator fields (plan dtype) the adjoint sweep fills for ``n_shots`` shots."""
        n = _lib.load().nw_adjoint_groups(C.byref(self.g), C.byref(self.tuning), n_shots)
        if n < 1:
            raise _lib.LibraryError(_lib.NW_ERR_ARG, "invalid adjoint group query")
        return n

    def shots_per_acc(self, n_shots: int) -> int:
        """Shots whose initial-state gradient term goes to one accumulator field (the adjoint's
        own grouping: adj_shots_per_cta in 2-D, one shot per field in 3-D)."""
        return int(self.tuning.adj_shots_per_cta) if self.g.ndim == 2 else 1

    # -- descriptors ------------------------------------------------------------------------
    def medium(self, c2dt2: torch.Tensor) -> _lib.Medium:
        m = _lib.Medium(c2dt2.data_ptr(), _lib.ptr(self.A), _lib.ptr(self.B))
        if self.pml is not None:
            m.pml_zz = self.pml["ZZ"].data_ptr()
            for ax in range(2):
                m.pml_alpha[ax] = self.pml["alpha"][ax].data_ptr()
                m.pml_beta[ax] = self.pml["beta"][ax].data_ptr()
                m.pml_half_inv_h[ax] = self.pml["half_inv_h"][ax]
            for k in range(4):
                m.pml_core[k] = self.pml["core"][k]
        return m

    def acquisition(self, n_shots: int, shot0: int = 0) -> _lib.Acquisition:
        a = _lib.Acquisition()
        a.n_shots = n_shots
        a.has_source = 1 if self.has_source else 0
        if self.has_source:
            a.src_corner = self.src_corner[shot0:].data_ptr()
            a.src_weight = self.src_weight[shot0:].data_ptr()
            a.wavelet = self.wavelet.data_ptr()
        a.n_rec = self.n_rec
        a.n_cells = self.n_cells
        a.rec_index = self.rec_index.data_ptr()
        a.rec_weight = self.rec_weight.data_ptr()
        a.cell_index = self.cell_index.data_ptr()
        a.cell_ptr = self.cell_ptr.data_ptr()
        a.cell_rec = self.cell_rec.data_ptr()
        a.cell_weight = self.cell_weight.data_ptr()
        if self.g.ndim == 2:
            a.tiles_z = self.tiles_z
            a.tile_rows, a.tile_cols = self.tile
            a.rec_corner = self.rec_corner.data_ptr()
            a.tile_rec_ptr = self.tile_rec_ptr.data_ptr()
            a.tile_rec_list = self.tile_rec_list.data_ptr()
            a.adj_tiles_z = self.adj_tiles_z
            a.adj_tile_rows, a.adj_tile_cols = self.adj_tile
            a.tile_cell_ptr = self.tile_cell_ptr.data_ptr()
            a.tile_cell_local = self.tile_cell_local.data_ptr()
            a.tile_cell_gid = self.tile_cell_gid.data_ptr()
            a.adj_tables_box = self.adj_tables_box
            a.adj_box_corner[0], a.adj_box_corner[1] = self.adj_box_corner
            if self.layer_cell_index is not None:
                a.n_layer_cells = int(self.layer_cell_index.numel())
                a.layer_cell_index = self.layer_cell_index.data_ptr()
                a.layer_cell_gid = self.layer_cell_gid.data_ptr()
        return a

    def empty_levels(self, n_levels: int, n_shots: int, zero: bool = True) -> torch.Tensor:
        fn = torch.zeros if zero else torch.empty
        return fn((n_levels, n_shots, self.field), device=self.device, dtype=self.dtype)

    def level_bytes(self, n_shots: int) -> int:
        return n_shots * self.field * torch.finfo(self.dtype).bits // 8

    def snapshot_bytes(self, n_shots: int, n_snap: int, kind: int) -> int:
        return int(_lib.load().nw_snapshot_bytes(C.byref(self.g), n_shots, n_snap, kind))


# ------------------------------------------------------------------------------------------------
# Binomial checkpointing over segments (the revolve strategy of Griewank and Walther, ACM TOMS 26
# (2000), "Algorithm 799: revolve", restated here for segments of K leapfrog steps). Reversing a
# segment is the recompute of its K Laplacian levels from its start state followed by its K adjoint
# steps; the start states live in snapshot slots. With fewer slots than segments, the adjoint re-runs
# parts of the forward sweep ("advances") to regenerate start states, taking new snapshots on the way.
# ------------------------------------------------------------------------------------------------
RESTORE, ADVANCE, TAKE, YOUTURN = 1, 2, 3, 4


def _beta(c: int, r: int) -> int:
    """Number of segments c slots can reverse with r advances per segment at most: C(c + r, c)."""
    return math.comb(c + r, c) if c >= 0 and r >= 0 else 0


def _repetitions(l: int, c: int) -> int:
    r = 0
    while _beta(c, r) < l:
        r += 1
    return r


def binomial_advances(l: int, c: int) -> int:
    """Fewest segment advances that reverse ``l`` segments with ``c`` slots, the first segment's start
    state in one of them: ``r l - C(c + r, c + 1)`` with ``r`` the least integer with
    ``C(c + r, c) >= l``. The first forward sweep is part of the count (it advances ``l - 1``)."""
    if l <= 1:
        return 0
    r = _repetitions(l, c)
    return r * l - _beta(c + 1, r - 1)


def binomial_schedule(n_seg: int, n_slots: int):
    """The binomial schedule of ``n_seg`` segments over ``n_slots`` snapshot slots.

    Returns ``(sweep_slot, actions)``: ``sweep_slot[j]`` is the slot the forward sweep encodes segment
    ``j``'s start state into (``-1``: none), and ``actions`` the adjoint's program, triples
    ``(RESTORE, slot, j)`` (decode a slot: the state at segment ``j``'s start), ``(ADVANCE, j0, j1)``
    (forward steps from segment ``j0``'s start to ``j1``'s), ``(TAKE, slot, j)`` (encode the state at
    segment ``j``'s start), ``(YOUTURN, j, 0)`` (recompute segment ``j``'s Laplacian levels from the
    state at its start, then its adjoint steps). Segments are reversed last to first.

    The recursion is revolve's: a subproblem of ``l`` segments whose first start state is in a slot,
    with ``c`` slots in all, puts its next snapshot ``m`` segments ahead, ``m`` the largest value of
    ``[max(l - C(c-1+r, c-1), C(c-2+r, c)), min(l - C(c-2+r, c-1), C(c-1+r, c))]`` (``r`` its
    repetition number), a range of optimal splits; with one slot it re-advances from its start for
    every segment. The first descent's snapshots are taken by the forward sweep, which then runs on to
    the last step for the traces; the first reversal therefore starts from a decoded snapshot, and if
    the descent ended inside a one-slot subproblem, the segments it advanced there are advanced again
    (``sweep_readvance``)."""
    if n_slots < 1 or n_seg < 1:
        raise ConfigError("binomial checkpointing needs at least one segment and one snapshot slot")
    sweep_slot = [-1] * n_seg
    actions: list[tuple[int, int, int]] = []
    free = list(range(n_slots - 1, 0, -1))  # slot 0 holds segment 0's start
    slot_of = {0: 0}
    st = {"cur": 0, "sweep": True}  # the segment start the ring holds (-1: none), and the sweep phase

    def reach(j):  # the ring to segment j's start: decode the nearest snapshot at or before j, advance
        if st["cur"] == j:
            return
        a = max(k for k in slot_of if k <= j)
        if st["cur"] < a or st["cur"] > j:
            actions.append((RESTORE, slot_of[a], a))
            st["cur"] = a
        if j > st["cur"]:
            actions.append((ADVANCE, st["cur"], j))
            st["cur"] = j

    def advance(a, b):
        if st["sweep"]:
            st["cur"] = b
        else:
            reach(a)
            reach(b)

    def take(j):
        k = free.pop()
        slot_of[j] = k
        if st["sweep"]:
            sweep_slot[j] = k
        else:
            reach(j)
            actions.append((TAKE, k, j))

    def youturn(j):
        if st["sweep"]:  # the sweep ran on to the end: the ring no longer holds any segment start
            st["sweep"] = False
            st["cur"] = -1
        reach(j)
        actions.append((YOUTURN, j, 0))
        st["cur"] = -1  # the recompute leaves the ring at the segment's end, which no one reverses next

    def reverse(a, b, c):
        l = b - a
        if l == 1:
            youturn(a)
            return
        if c == 1:
            for j in range(b - 1, a - 1, -1):
                advance(a, j)
                youturn(j)
            return
        r = _repetitions(l, c)
        lo = max(l - _beta(c - 1, r), _beta(c, r - 2), 1)
        hi = min(l - _beta(c - 1, r - 1), _beta(c, r - 1), l - 1)
        m = a + max(lo, hi)
        advance(a, m)
        take(m)
        reverse(m, b, c - 1)
        free.append(slot_of.pop(m))
        reverse(a, m, c)

    sweep_slot[0] = 0
    reverse(0, n_seg, n_slots)
    return sweep_slot, actions


def sweep_readvance(n_seg: int, n_slots: int) -> int:
    """Segments the first reversal re-advances because the forward sweep ran past its start: the length
    minus one of the one-slot subproblem the first descent ends in (0 when it ends on a snapshot)."""
    a, l, c = 0, n_seg, n_slots
    while l > 1 and c > 1:
        r = _repetitions(l, c)
        lo = max(l - _beta(c - 1, r), _beta(c, r - 2), 1)
        hi = min(l - _beta(c - 1, r - 1), _beta(c, r - 1), l - 1)
        m = max(lo, hi)
        a, l, c = a + m, l - m, c - 1
    return l - 1 if l > 1 else 0


def schedule_advances(n_seg: int, sweep_slot, actions) -> int:
    """Segment advances of a schedule: the forward sweep's ``n_seg - 1`` plus the adjoint's."""
    return n_seg - 1 + sum(b - a for op, a, b in actions if op == ADVANCE)


@functools.lru_cache(maxsize=64)
def cached_schedule(n_seg: int, n_slots: int):
    """``binomial_schedule`` as int32 triples for the library: ``(sweep_slot, program)``."""
    sweep_slot, actions = binomial_schedule(n_seg, n_slots)
    return (torch.tensor(sweep_slot, dtype=torch.int32),
            torch.tensor([v for a in actions for v in a] or [0], dtype=torch.int32))


def binomial_steps(n_steps: int, k: int, n_slots: int) -> int:
    """Forward steps of a binomial-checkpointed gradient: the sweep, each segment's recompute, and the
    adjoint's advances (``k`` steps each; the last segment may be shorter, which this ignores)."""
    n_seg = -(-n_steps // k)
    if n_slots >= n_seg:
        return 2 * n_steps
    extra = binomial_advances(n_seg, n_slots) - (n_seg - 1) + sweep_readvance(n_seg, n_slots)
    return 2 * n_steps + k * extra


def plan_storage(plan: DevicePlan, n_shots: int, n_steps: int, grad_mode: str,
                 checkpoint_every: int | None, snapshot: str, budget: int | None,
                 checkpoint_slots: int | None = None):
    """Choose the wavefield storage of a gradient run: ``("history",)``, ``("checkpoint", K)``
    (segments of ``K`` steps, a snapshot per segment start) or ``("checkpoint", K, slots)`` (binomial
    checkpointing of the segments over ``slots`` snapshot slots, fewer than the segments).

    ``grad_mode="autograd"`` keeps every level when it fits ``budget`` bytes and otherwise
    checkpoints; ``"checkpoint"`` uses segments of ``checkpoint_every`` steps (default
    ``ceil(sqrt(n_steps))``, the reference's choice) or the shortest segment whose storage fits the
    budget. When no segment length lets a snapshot per segment fit, the segment length and slot count
    that fit and need the fewest forward steps are chosen (binomial checkpointing, whose extra forward
    steps grow as the slots shrink). ``checkpoint_slots`` fixes the slot count.
    """
    lvl = plan.level_bytes(n_shots)
    hist = (n_steps + 3) * lvl  # n_steps Lap p levels and the pressure ring
    if grad_mode == "autograd" and (budget is None or hist <= budget) and not checkpoint_slots:
        return ("history", None)
    kind = _lib.SNAP_KINDS[snapshot]
    extra = 4 * lvl if plan.pml is not None else 0  # the PML's face fields
    snap1 = plan.snapshot_bytes(n_shots, 1, kind)

    def n_seg(k_):
        return -(-n_steps // k_)

    def cost(k_, slots=None):
        return snap1 * (n_seg(k_) if slots is None else slots) + (k_ + 3) * lvl + extra

    if checkpoint_slots:
        k = max(1, int(checkpoint_every)) if checkpoint_every else max(1, int(math.ceil(math.sqrt(max(1, n_steps)))))
        slots = max(1, int(checkpoint_slots))
        return ("checkpoint", k) if slots >= n_seg(k) else ("checkpoint", k, slots)
    if checkpoint_every:
        k = max(1, int(checkpoint_every))
        if budget is None or cost(k) <= budget:
            return ("checkpoint", k)
        ks = [k]
    else:
        k = max(1, int(math.ceil(math.sqrt(max(1, n_steps)))))
        if budget is None or cost(k) <= budget:
            return ("checkpoint", k)
        best = min(range(1, n_steps + 1), key=cost) if n_steps < 20000 else k
        if cost(best) <= budget:
            return ("checkpoint", best)
        ks = range(1, min(n_steps, 4096) + 1)
    # binomial checkpointing: for each segment length, the slots that fit; keep the fewest steps
    choice = None
    for k_ in ks:
        slots = (budget - (k_ + 3) * lvl - extra) // snap1 if budget is not None else 0
        if slots < 1:
            continue
        steps = binomial_steps(n_steps, k_, int(min(slots, n_seg(k_))))
        if choice is None or steps < choice[0]:
            choice = (steps, k_, int(min(slots, n_seg(k_))))
    if choice is None:
        raise ConfigError(
            f"checkpointed gradient needs at least {cost(1, 1) / 2**30:.1f} GiB, above the budget "
            f"{budget / 2**30:.1f} GiB; lower source_batch or use 16-bit snapshots")
    _, k, slots = choice
    return ("checkpoint", k) if slots >= n_seg(k) else ("checkpoint", k, slots)
