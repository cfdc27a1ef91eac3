"""``Projector``: prepared multiview projection as an ordinary PyTorch module.

Signature and behaviour follow the reference module (hcltech-robotics/dpt
``python/dpt/torch/modules.py:69-228``): ``Projector(*, grid, geometry,
precision="fp32", samples_per_ray=None, step_mm=None, anchor=None)`` and
``forward(field, pose=None, *, packed_pose=None, out=None)`` returning optical
depth ``(views, rows, columns)`` (FP32 for ``"fp32"``, FP64 for ``"fp64"``).
``pose`` is an FP64 right increment ``(6,)`` or ``(views, 6)`` about ``anchor``;
``packed_pose`` an explicit FP64 ``(12,)`` or ``(views, 12)`` pose.  Gradients
reach the field and either pose form (first order).  The default is 1024
midpoint samples; ``step_mm`` fixes the count once from the support diagonal.
"""

from __future__ import annotations

import math
from collections.abc import Sequence
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


def _samples(grid: GridSpec, samples_per_ray: int | None, step_mm: float | None) -> int:
    """Fixed midpoint count: explicit, default 1024, or ceil(support diagonal / step)."""
    if step_mm is None:
        return integer(1024 if samples_per_ray is None else samples_per_ray, "samples_per_ray",
                       minimum=1, maximum=2**31 - 1)
    if samples_per_ray is not None:
        raise ContractError("choose samples_per_ray or step_mm")
    step = finite_scalar(step_mm, "step_mm", minimum=0.0)
    if step == 0.0:
        raise ContractError("step_mm must be positive")
    nz, ny, nx = grid.shape
    diagonal = math.hypot(nx * grid.spacing_mm[0], ny * grid.spacing_mm[1], nz * grid.spacing_mm[2])
    count = diagonal / step
    if not math.isfinite(count) or count > 2**31 - 1:
        raise ContractError("step_mm requires too many midpoint samples")
    return max(1, math.ceil(count))


class Projector(torch.nn.Module):
    """Project device attenuation ``(nz, ny, nx)`` in mm^-1 to optical depth."""

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
        self.samples_per_ray = _samples(grid, samples_per_ray, step_mm)
        self.step_mm = step_mm
        self._configuration = _projection_ops.configuration(
            grid, self.geometry, self.samples_per_ray, "float32" if precision == "fp32" else "float64"
        )
        self._fixed_poses: dict[str, torch.Tensor] = {}
        if isinstance(anchor, torch.Tensor):
            self._check_pose(anchor, 12, "anchor")
            self._fixed_anchor = None
            if isinstance(anchor, torch.nn.Parameter):
                self.register_parameter("anchor", anchor)
            else:
                self.register_buffer("anchor", anchor)
        else:
            if anchor is not None and not isinstance(anchor, RigidTransform):
                raise ContractError("anchor must be a RigidTransform or FP64 packed Torch tensor")
            self._fixed_anchor = RigidTransform() if anchor is None else anchor
            self.register_buffer("anchor", None)

    @property
    def configuration(self) -> str:
        return self._configuration

    def _check_pose(self, value: torch.Tensor, components: int, name: str) -> None:
        shapes = ((components,), (len(self.geometry.views), components))
        if not isinstance(value, torch.Tensor) or value.dtype != torch.float64:
            raise ContractError(f"{name} must be a float64 Torch tensor")
        if tuple(value.shape) not in shapes:
            raise ContractError(f"{name} must have shape {shapes[0]} or {shapes[1]}")
        if not value.is_contiguous():
            raise ContractError(f"{name} must be contiguous")

    def _poses(self, field: torch.Tensor, pose: torch.Tensor | None,
               packed_pose: torch.Tensor | None) -> torch.Tensor:
        if packed_pose is not None:
            if pose is not None:
                raise ContractError("choose pose or packed_pose")
            self._check_pose(packed_pose, 12, "packed_pose")
            result = packed_pose
        else:
            anchor = self.anchor
            if anchor is None:
                key = str(field.device)
                if key not in self._fixed_poses:
                    assert self._fixed_anchor is not None
                    self._fixed_poses[key] = torch.tensor(
                        self._fixed_anchor.packed(), dtype=torch.float64, device=field.device
                    )
                anchor = self._fixed_poses[key]
            if anchor.device != field.device:
                raise ContractError("move the Projector anchor to the field device with .to(device)")
            self._check_pose(anchor, 12, "anchor")
            if pose is None:
                result = anchor
            else:
                self._check_pose(pose, 6, "pose")
                if pose.device != field.device:
                    raise ContractError("pose and field must share a device")
                result = compose_pose(anchor, pose)
        if result.device != field.device:
            raise ContractError("packed_pose and field must share a device")
        return result.expand(len(self.geometry.views), 12) if result.ndim == 1 else result

    def _check_output(self, out: torch.Tensor, field: torch.Tensor, poses: torch.Tensor) -> None:
        if not isinstance(out, torch.Tensor):
            raise ContractError("out must be a Torch tensor")
        dtype = torch.float64 if self.precision == "fp64" else torch.float32
        if tuple(out.shape) != self.geometry.shape or out.dtype != dtype or out.device != field.device:
            raise ContractError("out must match the projector's shape, dtype and input device")
        if not out.is_contiguous():
            raise ContractError("out must be contiguous")
        if out.requires_grad or (torch.is_grad_enabled() and (field.requires_grad or poses.requires_grad)):
            raise ContractError("out is an inference buffer; omit it for autograd or use torch.no_grad()")

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
        poses = self._poses(field, pose, packed_pose)
        if out is not None:
            self._check_output(out, field, poses)
            _projection_ops.project_out(field, poses, self._configuration, out)
            return out
        return _projection_ops.project(
            field,
            poses,
            self._configuration,
            field.requires_grad and torch.is_grad_enabled(),
            poses.requires_grad and torch.is_grad_enabled(),
        )
