"""ctypes binding of the projector's C ABI (``include/dpt_b200.h``).

The shared library ``dpt_b200/_lib/libdpt_b200.so`` is built in-tree by
``dpt_b200.build``.  There is no fallback: if the library is missing or cannot be
loaded, every projection call raises ``NativeLibraryError``.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

from .contracts import ContractError

LIBRARY_PATH = Path(__file__).resolve().parent / "_lib" / "libdpt_b200.so"
ABI_VERSION = 4
MAX_PACK = 64  # DPT_MAX_PACK: problems of one packed forward launch

# Mirrors of the header's enums.
F32, F64, F16, BF16 = 0, 1, 2, 3
ARITH_F32, ARITH_F64, ARITH_F32C, ARITH_MIXED, ARITH_FAST, ARITH_CELLS = 0, 1, 2, 3, 4, 5
DOMAIN_PHYSICAL, DOMAIN_SIGNED = 0, 1
RAYS_PANELS, RAYS_BUNDLE = 0, 1
PANEL_CONE, PANEL_PARALLEL, PANEL_CURVED = 0, 1, 2
VIEW_WORDS, VIEW_MODE_WORD = 20, 18
LAYOUT_REPLICATED, LAYOUT_DIRECT = 0, 1
VJP_VOLUME, VJP_POSE12, VJP_POSE6, VJP_PER_RAY6 = 1, 2, 4, 8
OUT_TRANSMISSION, OUT_COUNTS, OUT_LOG_TRANSMISSION, OUT_REMOVED = 1, 2, 4, 8
BEAM_NONE, BEAM_SCALAR, BEAM_DEVICE_SCALAR, BEAM_PER_PIXEL = 0, 1, 2, 3
CHECK_FINITE_NONNEGATIVE, CHECK_FINITE, CHECK_DECREMENT = 0, 1, 2
OBJECTIVE_SQUARED_ERROR, OBJECTIVE_POISSON = 0, 1

EXPORTS = (
    "dpt_b200_abi_version",
    "dpt_b200_error_string",
    "dpt_b200_packed_bytes",
    "dpt_b200_accumulator_bytes",
    "dpt_b200_pose_partials_bytes",
    "dpt_b200_prepare_field",
    "dpt_b200_forward",
    "dpt_b200_forward_packed",
    "dpt_b200_vjp",
    "dpt_b200_finish_pose",
    "dpt_b200_fold_volume",
    "dpt_b200_counts",
    "dpt_b200_pose_vjp_fixed",
    "dpt_b200_moments_bytes",
    "dpt_b200_forward_moments",
    "dpt_b200_pose_from_moments",
    "dpt_b200_gather_plan_bytes",
    "dpt_b200_gather_prepare",
    "dpt_b200_gather_count",
    "dpt_b200_gather",
    "dpt_b200_reduction_bytes",
    "dpt_b200_check_values",
    "dpt_b200_transmit",
    "dpt_b200_transmit_vjp",
    "dpt_b200_depth_from_removed",
    "dpt_b200_depth_from_removed_vjp",
    "dpt_b200_objective_check",
    "dpt_b200_objective",
    "dpt_b200_reduce_sum",
    "dpt_b200_read_probe",
)


class NativeLibraryError(RuntimeError):
    """The CUDA projector library is missing, stale or failed a call."""


class Problem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("views", ctypes.c_int32),
        ("rows", ctypes.c_int32),
        ("cols", ctypes.c_int32),
        ("samples", ctypes.c_int32),
        ("ray_kind", ctypes.c_int32),
        ("arith", ctypes.c_int32),
        ("field_dtype", ctypes.c_int32),
        ("image_dtype", ctypes.c_int32),
        ("layout", ctypes.c_int32),
        ("block_cols", ctypes.c_int32),
        ("field_domain", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("object_to_grid", ctypes.c_double * 9),
        ("grid_origin", ctypes.c_double * 3),
    ]


class Rays(ctypes.Structure):
    _fields_ = [
        ("poses", ctypes.c_void_p),
        ("view_table", ctypes.c_void_p),
        ("ray_sources", ctypes.c_void_p),
        ("ray_endpoints", ctypes.c_void_p),
        ("view_begin", ctypes.c_int32),
        ("view_count", ctypes.c_int32),
    ]


_P = ctypes.POINTER(Problem)
_R = ctypes.POINTER(Rays)
_V = ctypes.c_void_p
_I = ctypes.c_int32
_L = ctypes.c_int64
_F = ctypes.c_float
_D = ctypes.c_double

_SIGNATURES = {
    "dpt_b200_abi_version": ([], ctypes.c_int),
    "dpt_b200_error_string": ([ctypes.c_int], ctypes.c_char_p),
    "dpt_b200_packed_bytes": ([_P], ctypes.c_size_t),
    "dpt_b200_accumulator_bytes": ([_P], ctypes.c_size_t),
    "dpt_b200_pose_partials_bytes": ([_P, _I], ctypes.c_size_t),
    "dpt_b200_prepare_field": ([_P, _V, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_forward": ([_P, _R, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_forward_packed": ([_I, _P, _R, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_vjp": ([_P, _R, _V, _V, _I, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_finish_pose": ([_P, _I, _I, _I, _V, _V, _I, _V, _V], ctypes.c_int),
    "dpt_b200_fold_volume": ([_P, _V, _V, _I, _V, _I, _I, _V, _V], ctypes.c_int),
    "dpt_b200_counts": ([_P, _R, _V, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_pose_vjp_fixed": ([_P, _R, _V, _V, _I, _V, _V, _V], ctypes.c_int),
    "dpt_b200_moments_bytes": ([_P, _I], ctypes.c_size_t),
    "dpt_b200_forward_moments": ([_P, _R, _V, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_pose_from_moments": ([_P, _R, _V, _V, _I, _V, _V, _V], ctypes.c_int),
    "dpt_b200_gather_plan_bytes": ([_P, _I], ctypes.c_size_t),
    "dpt_b200_gather_prepare": ([_P, _R, _V, _V, _V], ctypes.c_int),
    "dpt_b200_gather_count": ([_P, _R, _V, _I, _V, _V], ctypes.c_int),
    "dpt_b200_gather": ([_P, _R, _V, _V, _V, _I, _I, _V, _V], ctypes.c_int),
    "dpt_b200_reduction_bytes": ([_L], ctypes.c_size_t),
    "dpt_b200_check_values": ([_V, _L, _I, _V, _V], ctypes.c_int),
    "dpt_b200_transmit": ([_V, _L, _I, _I, _V, _F, _V, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_transmit_vjp": (
        [_V, _L, _I, _V, _F, _V, _V, _V, _V, _V, _V, _V, _I, _V, _V], ctypes.c_int),
    "dpt_b200_depth_from_removed": ([_V, _L, _V, _V], ctypes.c_int),
    "dpt_b200_depth_from_removed_vjp": ([_V, _V, _L, _V, _I, _V, _V], ctypes.c_int),
    "dpt_b200_objective_check": ([_V, _I, _V, _V, _V, _L, _I, _I, _V, _V], ctypes.c_int),
    "dpt_b200_objective": (
        [_V, _I, _I, _V, _V, _V, _L, _I, _D, _D, _V, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_reduce_sum": ([_V, _L, _V, _V, _V, _V], ctypes.c_int),
    "dpt_b200_read_probe": ([_V, _L, _I, _V, _V], ctypes.c_int),
}

_lock = threading.Lock()
_library: ctypes.CDLL | None = None


def library() -> ctypes.CDLL:
    """Load (once) and return the CUDA library; raise if it is unavailable."""
    global _library
    if _library is not None:
        return _library
    with _lock:
        if _library is not None:
            return _library
        path = Path(os.environ.get("DPT_B200_LIBRARY", str(LIBRARY_PATH)))
        if not path.exists():
            raise NativeLibraryError(
                f"CUDA projector library not found at {path}; build it with "
                "`python -m dpt_b200.build`"
            )
        try:
            lib = ctypes.CDLL(str(path))
        except OSError as error:
            raise NativeLibraryError(f"cannot load {path}: {error}") from error
        for name, (argtypes, restype) in _SIGNATURES.items():
            function = getattr(lib, name)
            function.argtypes = argtypes
            function.restype = restype
        version = lib.dpt_b200_abi_version()
        if version != ABI_VERSION:
            raise NativeLibraryError(f"library ABI {version} does not match {ABI_VERSION}")
        _library = lib
        return lib


def check(code: int, what: str) -> None:
    """Raise for a nonzero return code of a C-ABI call."""
    if code == 0:
        return
    message = library().dpt_b200_error_string(code).decode()
    if code < 0:
        raise ContractError(f"{what}: {message}")
    raise NativeLibraryError(f"{what}: CUDA error {code}: {message}")
