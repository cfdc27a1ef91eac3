"""``project()``: the direct volume-to-optical-depth call.

Same signature and rules as the reference (hcltech-robotics/dpt
``python/dpt/api.py:18-98``): an ``ImagingVolume`` in mm^-1 is uploaded once as an
FP32 field and projected with a new ``Projector`` (default CUDA, FP32, 1024
samples); a device tensor is projected with ``prepared=Projector(...)``, keeping
its autograd graph.
"""

from __future__ import annotations

from typing import TYPE_CHECKING

from .contracts import ContractError
from .imaging import ImagingVolume

if TYPE_CHECKING:
    import torch

    from .torch.modules import GeometryInput, Precision, Projector

__all__ = ["project"]


def project(
    volume: ImagingVolume | torch.Tensor,
    geometry: GeometryInput | None = None,
    *,
    device: str | torch.device | None = None,
    precision: Precision | None = None,
    samples_per_ray: int | None = None,
    step_mm: float | None = None,
    pose: torch.Tensor | None = None,
    packed_pose: torch.Tensor | None = None,
    prepared: Projector | None = None,
    out: torch.Tensor | None = None,
) -> torch.Tensor:
    """Optical depth ``(views, rows, columns)`` on the device."""
    import torch

    from .plan import batched
    from .torch import Projector

    if prepared is not None and not isinstance(prepared, Projector):
        raise ContractError("prepared must be a dpt_b200.torch.Projector")
    if isinstance(volume, ImagingVolume):
        if volume.metadata.value_units != "mm^-1":
            raise ContractError("projection requires attenuation units='mm^-1'; convert HU first")
        grid = volume.grid
        field = torch.tensor(volume.values, dtype=torch.float32, device="cuda" if device is None else device)
    elif isinstance(volume, torch.Tensor):
        if prepared is None:
            raise ContractError("a device tensor requires prepared=Projector(grid=..., geometry=...)")
        grid = prepared.grid
        field = volume
        if device is not None:
            requested = torch.device(device)
            if not (requested == field.device or (requested.type == field.device.type and requested.index is None)):
                raise ContractError("device must match the supplied tensor; move it explicitly")
    else:
        raise ContractError("volume must be an ImagingVolume or a prepared device tensor")
    if prepared is None:
        if geometry is None:
            raise ContractError("geometry is required when no prepared Projector is supplied")
        prepared = Projector(grid=grid, geometry=geometry, precision="fp32" if precision is None else precision,
                             samples_per_ray=samples_per_ray, step_mm=step_mm)
    else:
        if grid != prepared.grid:
            raise ContractError("volume grid does not match the prepared Projector")
        if geometry is not None and batched(geometry) != prepared.geometry:
            raise ContractError("geometry does not match the prepared Projector")
        if precision is not None and precision != prepared.precision:
            raise ContractError("precision does not match the prepared Projector")
        if samples_per_ray is not None and samples_per_ray != prepared.samples_per_ray:
            raise ContractError("samples_per_ray does not match the prepared Projector")
        if step_mm is not None and step_mm != prepared.step_mm:
            raise ContractError("step_mm does not match the prepared Projector")
    return prepared(field, pose, packed_pose=packed_pose, out=out)
