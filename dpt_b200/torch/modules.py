"""``Projector``: prepared multiview projection as an ordinary PyTorch module.

Drop-in for the reference module (hcltech-robotics/dpt ``python/dpt/torch/modules.py:69-228``):
``Projector(*, grid, geometry, precision="fp32", samples_per_ray=None, step_mm=None,
anchor=None)`` and ``forward(field, pose=None, *, packed_pose=None, out=None)`` returning
optical depth ``(views, rows, columns)``, FP32 for ``"fp32"`` and FP64 for ``"fp64"``.

Argument rules (each violation raises ``ContractError`` with the message shown; rules are
checked top to bottom):

======================  =====================================================================
constructor
``grid``                a ``GridSpec`` -- "grid must be a GridSpec"
``precision``           ``"fp32"`` or ``"fp64"`` -- "precision must be fp32 or fp64"
sample count            ``samples_per_ray`` and ``step_mm`` exclusive -- "choose samples_per_ray
                        or step_mm"; a count is an int in [1, 2^31 - 1] (default 1024); a step
                        is finite, >= 0 and non-zero -- "step_mm must be positive"; the count it
                        implies, ceil(support diagonal / step), must be finite and below 2^31
                        -- "step_mm requires too many midpoint samples"
``anchor``              ``None`` (identity), a ``RigidTransform``, or an FP64 pose tensor (the
                        pose rule below, kept as a parameter when it is one, else a buffer) --
                        "anchor must be a RigidTransform or FP64 packed Torch tensor"
pose tensors            (``anchor`` 12, ``packed_pose`` 12, ``pose`` 6 components): an FP64
                        tensor -- "<name> must be a float64 Torch tensor"; shape (k,) or
                        (views, k) -- "<name> must have shape (k,) or (views, k)"; contiguous
                        -- "<name> must be contiguous"
forward
``field``               a tensor of the grid shape -- "field must be a Torch tensor with grid
                        shape (nz,ny,nx)"; contiguous FP32 (or FP16/BF16 for fp32 precision)
                        on a CUDA device
``packed_pose``         excludes ``pose`` -- "choose pose or packed_pose"; on the field's
                        device -- "packed_pose and field must share a device"
``pose``                an increment about the anchor; the anchor must be on the field's device
                        -- "move the Projector anchor to the field device with .to(device)";
                        the pose too -- "pose and field must share a device"
``out``                 a contiguous tensor of the image shape, dtype and device, never with
                        autograd -- "out must be a Torch tensor", "out must match the
                        projector's shape, dtype and input device", "out must be contiguous",
                        "out is an inference buffer; omit it for autograd or use
                        torch.no_grad()"
======================  =====================================================================
"""

from __future__ import annotations

import math
from collections.abc import Sequence
from dataclasses import dataclass
from typing import Literal

import torch

from ..contracts import ContractError, finite_scalar, integer
from ..geometry import BatchedGeometry, PanelGeometry, RigidTransform
from ..plan import batched
from ..volumes import GridSpec
from . import _projection_ops
from .geometry import compose_pose

Precision = Literal["fp32", "fp64"]
GeometryInput = BatchedGeometry | PanelGeometry | Sequence[PanelGeometry]

__all__ = ["Projector"]

DEFAULT_SAMPLES = 1024
MAX_SAMPLES = 2**31 - 1


def _sample_count(grid: GridSpec, samples_per_ray: int | None, step_mm: float | None) -> int:
    """The fixed midpoint count of every ray (sample count rules of the table above)."""
    if step_mm is not None and samples_per_ray is not None:
        raise ContractError("choose samples_per_ray or step_mm")
    if step_mm is None:
        chosen = DEFAULT_SAMPLES if samples_per_ray is None else samples_per_ray
        return integer(chosen, "samples_per_ray", minimum=1, maximum=MAX_SAMPLES)
    step = finite_scalar(step_mm, "step_mm", minimum=0.0)
    if not step > 0.0:
        raise ContractError("step_mm must be positive")
    # the support diagonal as the reference forms it (math.hypot), so a step gives its count
    extents = [n * h for n, h in zip(reversed(grid.shape), grid.spacing_mm, strict=True)]
    ratio = math.hypot(*extents) / step
    if not ratio <= MAX_SAMPLES:  # also rejects NaN and infinity
        raise ContractError("step_mm requires too many midpoint samples")
    return max(1, math.ceil(ratio))


@dataclass(frozen=True)
class _PoseRule:
    """Dtype, shape and layout rule of one pose tensor argument."""

    name: str
    components: int

    def check(self, value: object, views: int) -> torch.Tensor:
        if not isinstance(value, torch.Tensor) or value.dtype != torch.float64:
            raise ContractError(f"{self.name} must be a float64 Torch tensor")
        shared, per_view = (self.components,), (views, self.components)
        if tuple(value.shape) != shared and tuple(value.shape) != per_view:
            raise ContractError(f"{self.name} must have shape {shared} or {per_view}")
        if not value.is_contiguous():
            raise ContractError(f"{self.name} must be contiguous")
        return value


ANCHOR = _PoseRule("anchor", 12)
PACKED_POSE = _PoseRule("packed_pose", 12)
TANGENT = _PoseRule("pose", 6)


class _FixedAnchor:
    """A host ``RigidTransform`` anchor, materialised as a packed FP64 tensor once per device."""

    def __init__(self, transform: RigidTransform) -> None:
        self.transform = transform
        self._by_device: dict[torch.device, torch.Tensor] = {}

    def on(self, device: torch.device) -> torch.Tensor:
        packed = self._by_device.get(device)
        if packed is None:
            packed = torch.tensor(self.transform.packed(), dtype=torch.float64, device=device)
            self._by_device[device] = packed
        return packed


class Projector(torch.nn.Module):
    """Project device attenuation ``(nz, ny, nx)`` in mm^-1 to optical depth.

    ``pose`` is an FP64 right increment ``(6,)`` or ``(views, 6)`` about ``anchor``;
    ``packed_pose`` an explicit FP64 ``(12,)`` or ``(views, 12)`` pose (row-major rotation,
    then translation).  Gradients reach the field and either pose form (first order).  The
    default is 1024 midpoint samples; ``step_mm`` fixes the count once from the support
    diagonal.
    """

    anchor: torch.Tensor | None

    def __init__(
        self,
        *,
        grid: GridSpec,
        geometry: GeometryInput,
        precision: Precision = "fp32",
        samples_per_ray: int | None = None,
        step_mm: float | None = None,
        anchor: RigidTransform | torch.Tensor | None = None,
    ) -> None:
        super().__init__()
        if not isinstance(grid, GridSpec):
            raise ContractError("grid must be a GridSpec")
        if precision not in ("fp32", "fp64"):
            raise ContractError("precision must be fp32 or fp64")
        self.grid = grid
        self.geometry = batched(geometry)
        self.precision = precision
        self.samples_per_ray = _sample_count(grid, samples_per_ray, step_mm)
        self.step_mm = step_mm
        sampling = "float32" if precision == "fp32" else "float64"
        self._configuration = _projection_ops.configuration(grid, self.geometry, self.samples_per_ray, sampling)
        self._fixed_anchor: _FixedAnchor | None = None
        if isinstance(anchor, torch.Tensor):
            ANCHOR.check(anchor, self.views)
            # a Parameter is trained with the module, any other tensor follows it as a buffer
            register = self.register_parameter if isinstance(anchor, torch.nn.Parameter) else self.register_buffer
            register("anchor", anchor)
        elif anchor is None or isinstance(anchor, RigidTransform):
            self._fixed_anchor = _FixedAnchor(RigidTransform() if anchor is None else anchor)
            self.register_buffer("anchor", None)
        else:
            raise ContractError("anchor must be a RigidTransform or FP64 packed Torch tensor")

    @property
    def views(self) -> int:
        return len(self.geometry.views)

    @property
    def configuration(self) -> str:
        return self._configuration

    def _anchor_on(self, device: torch.device) -> torch.Tensor:
        if self.anchor is not None:
            return self.anchor
        assert self._fixed_anchor is not None
        return self._fixed_anchor.on(device)

    def _packed_poses(self, field: torch.Tensor, pose: torch.Tensor | None,
                      packed_pose: torch.Tensor | None) -> torch.Tensor:
        """The ``(views, 12)`` packed poses of this call (pose rules of the table above)."""
        if packed_pose is not None:
            if pose is not None:
                raise ContractError("choose pose or packed_pose")
            packed = PACKED_POSE.check(packed_pose, self.views)
        else:
            anchor = self._anchor_on(field.device)
            if anchor.device != field.device:
                raise ContractError("move the Projector anchor to the field device with .to(device)")
            ANCHOR.check(anchor, self.views)
            if pose is None:
                packed = anchor
            else:
                TANGENT.check(pose, self.views)
                if pose.device != field.device:
                    raise ContractError("pose and field must share a device")
                packed = compose_pose(anchor, pose)
        if packed.device != field.device:
            raise ContractError("packed_pose and field must share a device")
        return packed if packed.ndim == 2 else packed.expand(self.views, 12)

    def _require_output(self, out: object, field: torch.Tensor, poses: torch.Tensor) -> torch.Tensor:
        if not isinstance(out, torch.Tensor):
            raise ContractError("out must be a Torch tensor")
        expected = torch.float64 if self.precision == "fp64" else torch.float32
        if (tuple(out.shape), out.dtype, out.device) != (self.geometry.shape, expected, field.device):
            raise ContractError("out must match the projector's shape, dtype and input device")
        if not out.is_contiguous():
            raise ContractError("out must be contiguous")
        records_graph = torch.is_grad_enabled() and (field.requires_grad or poses.requires_grad)
        if out.requires_grad or records_graph:
            raise ContractError("out is an inference buffer; omit it for autograd or use torch.no_grad()")
        return out

    def forward(
        self,
        field: torch.Tensor,
        pose: torch.Tensor | None = None,
        *,
        packed_pose: torch.Tensor | None = None,
        out: torch.Tensor | None = None,
    ) -> torch.Tensor:
        """Optical depth with field and optional rigid-pose gradients."""
        if not isinstance(field, torch.Tensor) or tuple(field.shape) != self.grid.shape:
            raise ContractError("field must be a Torch tensor with grid shape (nz,ny,nx)")
        if field.dtype not in (torch.float32, torch.float16, torch.bfloat16) or not field.is_contiguous():
            raise ContractError("field must use contiguous float32 (or float16/bfloat16) storage")
        if field.dtype != torch.float32 and self.precision != "fp32":
            raise ContractError("FP16/BF16 fields require fp32 precision")
        if field.device.type != "cuda":
            raise ContractError("field must be on a CUDA device (the B200 projector has no CPU path)")
        poses = self._packed_poses(field, pose, packed_pose)
        if out is not None:
            _projection_ops.project_out(field, poses, self._configuration, self._require_output(out, field, poses))
            return out
        grad = torch.is_grad_enabled()
        return _projection_ops.project(field, poses, self._configuration, field.requires_grad and grad,
                                       poses.requires_grad and grad)
