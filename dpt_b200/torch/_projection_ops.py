"""Checked multiview Torch operators with one status checkpoint per call.

The operator names, schemas and behaviour follow the reference adapter
(hcltech-robotics/dpt ``python/dpt/torch/_projection_ops.py``):

* ``dpt::project(field, poses, value, active_volume, active_pose) -> Tensor``
  (``:256-264``), with a fake kernel for FakeTensor / ``torch.compile`` and a
  first-order autograd formula that calls
* ``dpt::project_vjp(field, poses, cotangent, value, active_volume, active_pose)
  -> (grad_field | empty(0), grad_poses | empty(0))`` (``:273-368``), and
* ``dpt::project_out(field, poses, value, out)`` for inference into caller
  storage (``:397-412``).

Only the immutable geometry crosses the dispatcher, as a canonical JSON string
(``configuration``, ``:41-58``).  Device workspaces are cached per (value,
device, stream, active flags), least recently used first out after 8 entries.
All three ops carry ``cudagraph_unsafe``: each call ends with a status readback.

Unlike the reference, the field may also be stored in FP16 or BF16 (``fp32``
precision only); its samples are then interpolated in FP32 with a compensated
ray sum, and its volume gradient is accumulated in FP32/FP64 and returned in the
field's dtype.  There is no CPU path: CPU tensors raise ``ContractError``.
"""

from __future__ import annotations

import json
from collections import OrderedDict
from dataclasses import asdict
from functools import lru_cache
from threading import RLock

import torch

from ..contracts import ContractError, integer
from ..geometry import BatchedGeometry, CurvedDetectorGeometry, DetectorGeometry, ParallelGeometry
from ..projection import ProjectionSpec, ProjectionWorkspace
from ..plan import plan_rays
from ..volumes import GridSpec

_CACHE_LIMIT = 8
_CACHE: OrderedDict[tuple, ProjectionWorkspace] = OrderedDict()
_CACHE_LOCK = RLock()
_TAGS = (torch.Tag.cudagraph_unsafe,)
_KINDS = {DetectorGeometry: "cone", ParallelGeometry: "parallel", CurvedDetectorGeometry: "curved"}
_CONSTRUCTORS = {"cone": DetectorGeometry, "parallel": ParallelGeometry, "curved": CurvedDetectorGeometry}
_FIELD_DTYPES = (torch.float32, torch.float16, torch.bfloat16)


def configuration(grid: GridSpec, geometry: BatchedGeometry, samples: int, precision: str) -> str:
    """Canonical JSON of the fixed physical configuration (no process-local handles)."""
    if precision not in ("float32", "float64"):
        raise ContractError("Torch projection arithmetic must be float32 or float64")
    return json.dumps(
        {
            "grid": asdict(grid),
            "views": [[_KINDS[type(panel)], asdict(panel)] for panel in geometry.views],
            "samples": samples,
            "precision": precision,
        },
        sort_keys=True,
        separators=(",", ":"),
        allow_nan=False,
    )


def _immutable(value):
    if isinstance(value, list):
        return tuple(_immutable(item) for item in value)
    return value


@lru_cache(maxsize=16)
def decode(value: str) -> tuple[GridSpec, BatchedGeometry, int, str]:
    encoded = json.loads(value)
    grid = GridSpec(**{key: _immutable(item) for key, item in encoded["grid"].items()})
    geometry = BatchedGeometry(
        tuple(
            _CONSTRUCTORS[kind](**{key: _immutable(item) for key, item in panel.items()})
            for kind, panel in encoded["views"]
        )
    )
    precision = encoded["precision"]
    if precision not in ("float32", "float64"):
        raise ContractError("Torch projection arithmetic must be float32 or float64")
    return grid, geometry, int(encoded["samples"]), precision


def _spec(precision: str, samples: int, field_dtype: torch.dtype, active_volume: bool,
          active_pose: bool) -> ProjectionSpec:
    if field_dtype == torch.float32:
        sampling, storage = precision, "float32"
    else:
        if precision != "float32":
            raise ContractError("FP16/BF16 fields require fp32 precision")
        sampling = "compensated"
        storage = "float16" if field_dtype == torch.float16 else "bfloat16"
    return ProjectionSpec(samples, active_pose=active_pose, active_volume=active_volume,
                          precision=precision, sampling_precision=sampling,
                          storage_precision=storage)


def workspace(field: torch.Tensor, value: str, active_volume: bool, active_pose: bool) -> ProjectionWorkspace:
    """The cached workspace for this configuration on the field's device and stream."""
    stream = torch.cuda.current_stream(field.device).cuda_stream
    key = (value, str(field.device), stream, field.dtype, active_volume, active_pose)
    with _CACHE_LOCK:
        found = _CACHE.get(key)
        if found is not None:
            _CACHE.move_to_end(key)
            return found
        grid, geometry, samples, precision = decode(value)
        spec = _spec(precision, samples, field.dtype, active_volume, active_pose)
        found = ProjectionWorkspace(plan_rays(grid, geometry), spec, field.device)
        _CACHE[key] = found
        while len(_CACHE) > _CACHE_LIMIT:
            _CACHE.popitem(last=False)
        return found


def set_cache_limit(limit: int) -> None:
    """Keep up to ``limit`` workspaces (plans, field copies, scratch) across calls; the least
    recently used beyond it are released.  The default, 8, suits one training loop; callers
    cycling through many configurations keep their state warm with a larger limit."""
    global _CACHE_LIMIT
    integer(limit, "limit", minimum=1)
    with _CACHE_LOCK:
        _CACHE_LIMIT = limit
        while len(_CACHE) > _CACHE_LIMIT:
            _CACHE.popitem(last=False)


def clear_cache() -> None:
    with _CACHE_LOCK:
        _CACHE.clear()


def metadata(field: torch.Tensor, poses: torch.Tensor, value: str) -> tuple[tuple[int, ...], torch.dtype]:
    grid, geometry, _, precision = decode(value)
    if (
        tuple(field.shape) != grid.shape
        or field.dtype not in _FIELD_DTYPES
        or not field.is_contiguous()
    ):
        raise ContractError("field must use contiguous float32/float16/bfloat16 storage with grid shape")
    if field.dtype != torch.float32 and precision != "float32":
        raise ContractError("FP16/BF16 fields require fp32 precision")
    if (
        tuple(poses.shape) != (len(geometry.views), 12)
        or poses.dtype != torch.float64
        or poses.device != field.device
    ):
        raise ContractError("poses must be float64 (views,12) on the field device")
    return geometry.shape, torch.float64 if precision == "float64" else torch.float32


def _require_cuda(field: torch.Tensor) -> None:
    if field.device.type != "cuda":
        raise ContractError("the B200 projector requires CUDA tensors (there is no CPU path)")


def _forward(field, poses, value, active_volume, active_pose, out=None):
    shape, dtype = metadata(field, poses, value)
    _require_cuda(field)
    if out is not None and (
        tuple(out.shape) != shape or out.dtype != dtype or out.device != field.device
        or not out.is_contiguous()
    ):
        raise ContractError("out must match the projector's shape, dtype and input device")
    if out is not None and any(
        out.untyped_storage().data_ptr() == x.untyped_storage().data_ptr() for x in (field, poses)
    ):
        raise ContractError("out must not share storage with projection inputs")
    entry = workspace(field, value, active_volume, active_pose)
    with torch.no_grad():
        # a pose that will be differentiated: where the arithmetic prefers it, gather the pose
        # moments in this pass, so the backward's pose VJP needs no second sampling pass
        # (results are unchanged either way)
        return entry.forward(field, poses.contiguous(), out,
                             moments=active_pose and out is None and entry.moments_preferred())


@torch.library.custom_op("dpt::project", mutates_args=(), tags=_TAGS)
def project(
    field: torch.Tensor, poses: torch.Tensor, value: str, active_volume: bool, active_pose: bool
) -> torch.Tensor:
    return _forward(field, poses, value, active_volume, active_pose)


@project.register_fake
def _project_fake(field, poses, value, active_volume, active_pose):
    shape, dtype = metadata(field, poses, value)
    return torch.empty(shape, dtype=dtype, device=field.device)


@torch.library.custom_op("dpt::project_vjp", mutates_args=(), tags=_TAGS)
def project_vjp(
    field: torch.Tensor,
    poses: torch.Tensor,
    cotangent: torch.Tensor,
    value: str,
    active_volume: bool,
    active_pose: bool,
) -> tuple[torch.Tensor, torch.Tensor]:
    shape, dtype = metadata(field, poses, value)
    if tuple(cotangent.shape) != shape or cotangent.dtype != dtype or cotangent.device != field.device:
        raise ContractError("cotangent must match the projected image shape, dtype and device")
    if not active_volume and not active_pose:
        raise ContractError("request at least one projection gradient")
    _require_cuda(field)
    entry = workspace(field, value, active_volume, active_pose)
    with torch.no_grad():
        gradient, pose_gradient = entry.vjp(
            field, poses.contiguous(), cotangent, volume=active_volume,
            pose="matrix" if active_pose else None, volume_dtype=torch.float32,
        )
    if gradient is None:
        gradient = field.new_empty((0,))
    elif gradient.dtype != field.dtype:
        gradient = gradient.to(field.dtype)
    if pose_gradient is None:
        pose_gradient = poses.new_empty((0,))
    return gradient, pose_gradient


@project_vjp.register_fake
def _vjp_fake(field, poses, cotangent, value, active_volume, active_pose):
    shape, dtype = metadata(field, poses, value)
    if tuple(cotangent.shape) != shape or cotangent.dtype != dtype or cotangent.device != field.device:
        raise ContractError("cotangent must match the projected image shape, dtype and device")
    return (
        field.new_empty(field.shape if active_volume else (0,)),
        poses.new_empty(poses.shape if active_pose else (0,)),
    )


def _setup_context(ctx, inputs, output):
    field, poses, value, _, _ = inputs
    ctx.save_for_backward(field, poses)
    ctx.configuration = value


def _backward(ctx, cotangent):
    if torch.is_grad_enabled():
        raise ContractError("the Torch projection adapter supports first-order derivatives only")
    field, poses = ctx.saved_tensors
    active_volume, active_pose = ctx.needs_input_grad[:2]
    gradient, pose_gradient = project_vjp(
        field, poses, cotangent.contiguous(), ctx.configuration, active_volume, active_pose
    )
    return (
        gradient if active_volume else None,
        pose_gradient if active_pose else None,
        None,
        None,
        None,
    )


project.register_autograd(_backward, setup_context=_setup_context)


@torch.library.custom_op("dpt::project_out", mutates_args={"out"}, tags=_TAGS)
def project_out(field: torch.Tensor, poses: torch.Tensor, value: str, out: torch.Tensor) -> None:
    _forward(field, poses, value, False, False, out)


@project_out.register_fake
def _out_fake(field, poses, value, out):
    shape, dtype = metadata(field, poses, value)
    if tuple(out.shape) != shape or out.dtype != dtype or out.device != field.device or not out.is_contiguous():
        raise ContractError("out must match the projector's shape, dtype and input device")
