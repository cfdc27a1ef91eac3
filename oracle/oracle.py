"""ctypes wrapper of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Functions take a ``RayPlan``-like object (attributes ``views, rows, cols,
ray_kind, object_to_grid, grid_origin, view_table, sources, endpoints`` and
``grid.shape``) plus numpy arrays, and return numpy arrays.  The ``dpt_problem``
structure is declared here independently of the product's binding so that a
layout mistake on either side shows up as a disagreement.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import build as _build

F32, F64, F16, BF16 = 0, 1, 2, 3
ARITH_F32, ARITH_F64, ARITH_F32C, ARITH_MIXED, ARITH_FAST, ARITH_CELLS = 0, 1, 2, 3, 4, 5
RAYS_PANELS, RAYS_BUNDLE = 0, 1
VJP_VOLUME, VJP_POSE12, VJP_POSE6, VJP_PER_RAY6 = 1, 2, 4, 8


class _Problem(ctypes.Structure):
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


_lib = None


def library():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(_build.build()))
        P, V = ctypes.POINTER(_Problem), ctypes.c_void_p
        lib.oracle_forward.argtypes = [P, V, V, V, V, V, V, V, ctypes.c_int]
        lib.oracle_forward.restype = ctypes.c_int
        lib.oracle_counts.argtypes = [P, V, V, V, V, V, V, V, ctypes.c_int]
        lib.oracle_counts.restype = ctypes.c_int
        lib.oracle_vjp.argtypes = [P, V, V, V, V, V, V, ctypes.c_int32, V, V, V, ctypes.c_int]
        lib.oracle_vjp.restype = ctypes.c_int
        lib.oracle_check_field.argtypes = [P, V, ctypes.c_int64]
        lib.oracle_check_field.restype = ctypes.c_int
        lib.oracle_check_pose.argtypes = [V]
        lib.oracle_check_pose.restype = ctypes.c_int
        lib.oracle_gather.argtypes = [P, V, V, V, V, V, V, ctypes.c_int, ctypes.c_int, V, ctypes.c_int]
        lib.oracle_gather.restype = ctypes.c_int
        lib.oracle_gather_cells.argtypes = lib.oracle_gather.argtypes
        lib.oracle_gather_cells.restype = ctypes.c_int
        _lib = lib
    return _lib


def _ptr(array: np.ndarray | None) -> int | None:
    return None if array is None else array.ctypes.data


@dataclass
class OracleCall:
    problem: _Problem
    poses: np.ndarray
    table: np.ndarray | None
    sources: np.ndarray | None
    endpoints: np.ndarray | None


def _call(plan, samples: int, arith: int, field_dtype: int, image_dtype: int, poses) -> OracleCall:
    nz, ny, nx = plan.grid.shape
    p = _Problem()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.views, p.rows, p.cols = plan.views, plan.rows, plan.cols
    p.samples, p.ray_kind, p.arith = samples, plan.ray_kind, arith
    p.field_dtype, p.image_dtype, p.layout = field_dtype, image_dtype, 0
    for k in range(9):
        p.object_to_grid[k] = plan.object_to_grid[k]
    for k in range(3):
        p.grid_origin[k] = plan.grid_origin[k]
    poses = np.ascontiguousarray(np.broadcast_to(np.asarray(poses, dtype=np.float64).reshape(-1, 12),
                                                 (plan.views, 12)))
    table = None if plan.view_table is None else np.ascontiguousarray(plan.view_table, dtype=np.float64)
    sources = None if plan.sources is None else np.ascontiguousarray(plan.sources, dtype=np.float64)
    endpoints = None if plan.endpoints is None else np.ascontiguousarray(plan.endpoints, dtype=np.float64)
    return OracleCall(p, poses, table, sources, endpoints)


def _field_array(field: np.ndarray, field_dtype: int) -> np.ndarray:
    if field_dtype == F32:
        return np.ascontiguousarray(field, dtype=np.float32).reshape(-1)
    # half storage passed as raw 16-bit patterns
    return np.ascontiguousarray(field).view(np.uint16).reshape(-1)


def forward(plan, field, poses, *, samples: int, arith: int = ARITH_F32, field_dtype: int = F32,
            image_dtype: int = F32, threads: int = 0):
    """Optical depth of every ray (flat, view-major) and the per-view status words."""
    call = _call(plan, samples, arith, field_dtype, image_dtype, poses)
    data = _field_array(field, field_dtype)
    image = np.zeros(plan.views * plan.rows * plan.cols, dtype=np.float64 if image_dtype == F64 else np.float32)
    status = np.zeros(plan.views, dtype=np.int32)
    code = library().oracle_forward(
        ctypes.byref(call.problem), _ptr(call.poses), _ptr(call.table), _ptr(call.sources),
        _ptr(call.endpoints), _ptr(data), _ptr(image), _ptr(status), threads,
    )
    assert code == 0
    return image, status


def counts(plan, poses, *, samples: int, arith: int = ARITH_F32, threads: int = 0):
    """Per-ray clip interval (lower, upper) and number of midpoints inside the support."""
    call = _call(plan, samples, arith, F32, F32, poses)
    n = plan.views * plan.rows * plan.cols
    lower, upper = np.zeros(n), np.zeros(n)
    realised = np.zeros(n, dtype=np.int32)
    code = library().oracle_counts(
        ctypes.byref(call.problem), _ptr(call.poses), _ptr(call.table), _ptr(call.sources),
        _ptr(call.endpoints), _ptr(lower), _ptr(upper), _ptr(realised), threads,
    )
    assert code == 0
    return lower, upper, realised


def vjp(plan, field, poses, cotangent, *, samples: int, flags: int, arith: int = ARITH_F32,
        field_dtype: int = F32, image_dtype: int = F32, threads: int = 0):
    """Volume gradient (FP64, voxels), pose gradient and status words of the joint VJP."""
    call = _call(plan, samples, arith, field_dtype, image_dtype, poses)
    data = _field_array(field, field_dtype)
    seed = np.ascontiguousarray(cotangent, dtype=np.float64 if image_dtype == F64 else np.float32).reshape(-1)
    voxels = int(np.prod(plan.grid.shape))
    volume = np.zeros(voxels, dtype=np.float64)
    if flags & VJP_PER_RAY6:
        pose = np.zeros((plan.views * plan.rows * plan.cols, 6))
    elif flags & VJP_POSE12:
        pose = np.zeros((plan.views, 12))
    else:
        pose = np.zeros((plan.views, 6))
    status = np.zeros(plan.views, dtype=np.int32)
    code = library().oracle_vjp(
        ctypes.byref(call.problem), _ptr(call.poses), _ptr(call.table), _ptr(call.sources),
        _ptr(call.endpoints), _ptr(data), _ptr(seed), flags, _ptr(volume), _ptr(pose),
        _ptr(status), threads,
    )
    assert code == 0
    return volume, pose, status


def gather(plan, poses, cotangent, *, samples: int, image_dtype: int = F64, out_dtype: int = F64,
           out=None, accumulate: bool = False, cells: bool = False, threads: int = 0):
    """Deterministic all-ray adjoint gather of the strict FP64 midpoint operator (or, with
    ``cells``, of cell-Gauss integration): per voxel, views ascending, all rays and samples (or
    cell segments) in order.  Returns (volume, status bit word)."""
    call = _call(plan, samples, ARITH_CELLS if cells else ARITH_F64, F32, image_dtype, poses)
    seed = np.ascontiguousarray(cotangent, dtype=np.float64 if image_dtype == F64 else np.float32).reshape(-1)
    voxels = int(np.prod(plan.grid.shape))
    dtype = np.float64 if out_dtype == F64 else np.float32
    volume = np.zeros(voxels, dtype=dtype) if out is None else np.ascontiguousarray(out, dtype=dtype).reshape(-1).copy()
    status = np.zeros(1, dtype=np.int32)
    function = library().oracle_gather_cells if cells else library().oracle_gather
    code = function(
        ctypes.byref(call.problem), _ptr(call.poses), _ptr(call.table), _ptr(call.sources),
        _ptr(call.endpoints), _ptr(seed), _ptr(volume), out_dtype, int(accumulate), _ptr(status), threads,
    )
    assert code == 0
    return volume, int(status[0])


def check_field(field: np.ndarray, field_dtype: int = F32, domain: int = 0) -> int:
    p = _Problem()
    p.field_dtype = field_dtype
    p.field_domain = domain
    data = _field_array(field, field_dtype)
    return library().oracle_check_field(ctypes.byref(p), _ptr(data), data.size)


def check_pose(pose) -> int:
    pose = np.ascontiguousarray(pose, dtype=np.float64)
    return library().oracle_check_pose(_ptr(pose))
