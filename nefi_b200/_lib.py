"""ctypes binding of the C ABI in ``include/nefi_wave.h`` (the in-tree ``libnefiwave.so``).

Structures mirror the header field by field. Device buffers are passed as raw pointers taken from
torch tensors (``Tensor.data_ptr()``) and work is enqueued on the caller's current CUDA stream.
Loading fails loudly when the library is missing: there is no CPU or eager fallback.
"""

from __future__ import annotations

import ctypes as C
import functools
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "libnefiwave.so"
ABI_VERSION = 6

NW_F32, NW_F64 = 0, 1
NW_ABS_NONE, NW_ABS_SPONGE, NW_ABS_CERJAN, NW_ABS_PML = 0, 1, 2, 3
NW_SNAP_EXACT, NW_SNAP_F16, NW_SNAP_BF16 = 0, 1, 2
NW_OK, NW_ERR_ARG, NW_ERR_CUDA, NW_ERR_UNSUPPORTED, NW_ERR_NONFINITE, NW_ERR_TIMEOUT = range(6)
NW_SNAP_BLOCK = 32

NW_SNAP_I16 = 3
NW_SNAP_D16 = 4
SNAP_KINDS = {"exact": NW_SNAP_EXACT, "fp16": NW_SNAP_F16, "bf16": NW_SNAP_BF16, "fixed16": NW_SNAP_I16,
              "delta16": NW_SNAP_D16}


class Grid(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32), ("order", C.c_int32), ("dtype", C.c_int32), ("absorbing", C.c_int32),
        ("n", C.c_int32 * 3), ("core_lo", C.c_int32 * 3), ("core_hi", C.c_int32 * 3),
        ("w_center", C.c_double), ("w1", C.c_double * 3), ("w2", C.c_double * 3),
        ("radius", C.c_int32), ("guard", C.c_int32),
        ("stride", C.c_int64 * 3), ("origin", C.c_int64), ("field_elems", C.c_int64),
    ]


class Tuning(C.Structure):
    _fields_ = [("vz", C.c_int32), ("rx", C.c_int32), ("shots_per_cta", C.c_int32),
                ("adj_vz", C.c_int32), ("adj_rx", C.c_int32), ("adj_shots_per_cta", C.c_int32),
                ("depth", C.c_int32), ("reserved", C.c_int32)]


class Acquisition(C.Structure):
    _fields_ = [
        ("n_shots", C.c_int32), ("has_source", C.c_int32),
        ("src_corner", C.c_void_p), ("src_weight", C.c_void_p), ("wavelet", C.c_void_p),
        ("n_rec", C.c_int32), ("n_cells", C.c_int32),
        ("rec_index", C.c_void_p), ("rec_weight", C.c_void_p),
        ("cell_index", C.c_void_p), ("cell_ptr", C.c_void_p), ("cell_rec", C.c_void_p),
        ("cell_weight", C.c_void_p),
        ("tiles_z", C.c_int32), ("tile_rows", C.c_int32), ("tile_cols", C.c_int32),
        ("rec_corner", C.c_void_p), ("tile_rec_ptr", C.c_void_p), ("tile_rec_list", C.c_void_p),
        ("adj_tiles_z", C.c_int32), ("adj_tile_rows", C.c_int32), ("adj_tile_cols", C.c_int32),
        ("tile_cell_ptr", C.c_void_p), ("tile_cell_local", C.c_void_p), ("tile_cell_gid", C.c_void_p),
        ("adj_tables_box", C.c_int32), ("adj_box_corner", C.c_int32 * 2),
        ("n_layer_cells", C.c_int32), ("layer_cell_index", C.c_void_p), ("layer_cell_gid", C.c_void_p),
    ]


class Medium(C.Structure):
    _fields_ = [("c2dt2", C.c_void_p), ("coef_a", C.c_void_p), ("coef_b", C.c_void_p),
                ("pml_zz", C.c_void_p), ("pml_alpha", C.c_void_p * 2), ("pml_beta", C.c_void_p * 2),
                ("pml_half_inv_h", C.c_double * 2), ("pml_core", C.c_int32 * 4)]


class Time(C.Structure):
    _fields_ = [("n_steps", C.c_int32), ("substeps", C.c_int32), ("n_t", C.c_int32),
                ("first_b_one", C.c_int32)]


class Storage(C.Structure):
    _fields_ = [("history", C.c_void_p), ("ring", C.c_void_p), ("snap", C.c_void_p),
                ("segbuf", C.c_void_p), ("segment", C.c_int32), ("snap_kind", C.c_int32),
                ("pml_psi", C.c_void_p), ("snap_slot", C.c_void_p), ("schedule", C.c_void_p),
                ("n_schedule", C.c_int32), ("ring_levels", C.c_int32)]


class BatchProblem(C.Structure):
    _fields_ = [("grid", Grid), ("medium", Medium), ("acq", Acquisition), ("time", Time),
                ("storage", Storage), ("work", C.c_void_p), ("grad_acc", C.c_void_p),
                ("traces", C.c_void_p), ("grad_traces", C.c_void_p)]


class Traces(C.Structure):
    _fields_ = [("dtype", C.c_int32), ("n_t", C.c_int32), ("n_traces", C.c_int64), ("mask", C.c_void_p),
                ("mask_per_sample", C.c_int32), ("log2_len", C.c_int32)]


NW_FILTER_LOWPASS, NW_FILTER_GAUSSIAN = 0, 1
NW_MISFIT_STATE, NW_MISFIT_COUNT, NW_MISFIT_DEN, NW_MISFIT_SCALE, NW_MISFIT_SUM, NW_MISFIT_LOSS = (
    2056, 2048, 2049, 2050, 2051, 2052)

P = C.POINTER
VP = C.c_void_p
_SIGNATURES = {
    "nw_abi_version": (C.c_int, []),
    "nw_built_arch": (C.c_int, []),
    "nw_last_error": (C.c_char_p, []),
    "nw_grid_layout": (C.c_int, [P(Grid)]),
    "nw_snapshot_bytes": (C.c_size_t, [P(Grid), C.c_int32, C.c_int32, C.c_int32]),
    "nw_prepare_medium": (C.c_int, [P(Grid), VP, VP, C.c_double, VP, VP]),
    "nw_initial_state": (C.c_int, [P(Grid), VP, P(Medium), C.c_int32, VP, VP, VP, VP]),
    "nw_tile_shape": (C.c_int, [P(Grid), P(Tuning), P(C.c_int32)]),
    "nw_adjoint_groups": (C.c_int, [P(Grid), P(Tuning), C.c_int32]),
    "nw_forward": (C.c_int, [P(Grid), P(Medium), P(Acquisition), P(Time), P(Storage), P(Tuning),
                             C.c_int32, C.c_int32, VP, VP]),
    "nw_adjoint": (C.c_int, [P(Grid), P(Medium), P(Acquisition), P(Time), P(Storage), P(Tuning), VP,
                             VP, VP, VP, VP, VP]),
    "nw_reduce_grad_c": (C.c_int, [P(Grid), VP, VP, C.c_double, C.c_int32, VP, C.c_int32, VP, VP]),
    "nw_initial_state_adjoint": (C.c_int, [P(Grid), VP, P(Medium), P(Time), C.c_int32, VP, VP, VP,
                                           VP, VP, C.c_int32, VP]),
    "nw_sample": (C.c_int, [P(Grid), P(Acquisition), C.c_int32, VP, C.c_int32, VP, VP]),
    "nw_status": (C.c_int, [VP]),
    "nw_zero_ghosts": (C.c_int, [P(Grid), VP, C.c_int64, VP]),
    "nw_adjoint_grad_c_noalloc": (C.c_int, [P(Grid), VP, P(Medium), P(Acquisition), P(Time), P(Storage),
                                            P(Tuning), VP, C.c_double, VP, VP, VP]),
    "nw_launch_count": (C.c_uint64, []),
    "nw_time_reversal": (C.c_int, [P(Grid), P(Medium), P(Acquisition), P(Time), P(Storage), P(Tuning), VP,
                                   C.c_int32, VP, VP]),
    "nw_filter_log2_len": (C.c_int, [C.c_int32]),
    "nw_filter_response": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32, VP]),
    "nw_trace_filter": (C.c_int, [P(Traces), VP, VP, VP, VP]),
    "nw_misfit_prepare": (C.c_int, [P(Traces), VP, VP, C.c_int32, VP, VP]),
    "nw_misfit": (C.c_int, [P(Traces), VP, VP, VP, VP, VP, VP, VP]),
    "nw_batch_table_bytes": (C.c_size_t, [C.c_int32]),
    "nw_batch_prepare": (C.c_int, [P(BatchProblem), C.c_int32, P(Tuning), VP, VP]),
    "nw_batch_forward": (C.c_int, [P(BatchProblem), C.c_int32, P(Tuning), VP, VP]),
    "nw_batch_adjoint": (C.c_int, [P(BatchProblem), C.c_int32, P(Tuning), VP, VP]),
}
EXPORTED = tuple(_SIGNATURES)

_lib: C.CDLL | None = None


class LibraryError(RuntimeError):
    """The CUDA library is missing, fails to load or reported an error."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libnefiwave error {code}: {msg}")
        self.code = code


def load(path: Path | None = None) -> C.CDLL:
    """Load (once) and return the library; raises ``LibraryError`` if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise LibraryError(-1, f"{p} is missing; build it with `python -m nefi_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.nw_abi_version() != ABI_VERSION:
        raise LibraryError(-1, f"ABI version mismatch: {lib.nw_abi_version()}")
    if path is None:
        _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != NW_OK:
        msg = load().nw_last_error().decode(errors="replace")
        raise LibraryError(rc, msg)


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _cuda_device(v) -> torch.device | None:
    if isinstance(v, torch.Tensor):
        return v.device if v.is_cuda else None
    if isinstance(v, str) and v.startswith("cuda"):
        return torch.device(v)
    if isinstance(v, torch.device):
        return v if v.type == "cuda" else None
    d = getattr(v, "device", None)
    return d if isinstance(d, torch.device) and d.type == "cuda" else None


def on_device(fn):
    """Run ``fn`` with the current CUDA device set to the device of its first CUDA tensor argument
    (else of its first argument naming a CUDA device, or holding one as ``.device``). The library
    launches on the current device and the side streams it keeps are per device, so a call whose
    tensors live on another GPU than the current one runs there instead of failing or mixing devices."""

    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        vals = (*args, *kwargs.values())
        dev = next((v.device for v in vals if isinstance(v, torch.Tensor) and v.is_cuda), None)
        if dev is None:
            dev = next((d for d in map(_cuda_device, vals) if d is not None), None)
        if dev is None:
            return fn(*args, **kwargs)
        with torch.cuda.device(dev):
            return fn(*args, **kwargs)

    return wrapper


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return NW_F32
    if dtype == torch.float64:
        return NW_F64
    raise TypeError(f"unsupported dtype {dtype}; use float32 or float64")
