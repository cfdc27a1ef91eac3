"""Imaging volumes and the conversions on the projection path.

``ImagingVolume`` / ``ImagingMetadata`` keep the fields the projector reads from
the reference's records (hcltech-robotics/dpt ``python/dpt/imaging_io.py:44-160``);
file readers (NIfTI / DICOM) are not part of this package.
``ct_to_attenuation`` and ``standard_views`` follow ``python/dpt/imaging.py:112-187``.
"""

from __future__ import annotations

import math
from collections.abc import Sequence
from dataclasses import dataclass, replace
from typing import Any, Literal

import numpy as np

from .contracts import ContractError, finite_scalar
from .geometry import BatchedGeometry, ConeBeamIntrinsics
from .volumes import GridSpec

WATER_60KEV_MM = 0.02059  # NIST water mass attenuation at 60 keV (0.2059 cm^2/g) at 1 g/cm^3


@dataclass(frozen=True, slots=True)
class ImagingMetadata:
    """Provenance and units of ``values[z, y, x]``; spatial lengths are mm."""

    source_format: Literal["nifti", "dicom", "synthetic"]
    coordinate_frame: Literal["RAS", "LPS", "synthetic"]
    value_units: str
    measurement_unit_code: Any = None

    def __post_init__(self) -> None:
        if not isinstance(self.value_units, str) or not self.value_units.strip():
            raise ContractError("value_units must be a non-empty unit label")


@dataclass(frozen=True, slots=True)
class ImagingVolume:
    """Finite real values of shape ``grid.shape`` (x fastest), read-only copy."""

    values: Any
    grid: GridSpec
    metadata: ImagingMetadata

    def __post_init__(self) -> None:
        raw = np.asarray(self.values)
        if raw.dtype.kind not in "biuf":
            raise ContractError("imaging values must be real")
        values = np.array(raw, order="C", copy=True)
        if tuple(values.shape) != self.grid.shape:
            raise ContractError("imaging values must have grid shape (nz,ny,nx)")
        if not np.isfinite(values).all():
            raise ContractError("imaging values must be finite")
        values.flags.writeable = False
        object.__setattr__(self, "values", values)

    @property
    def shape(self) -> tuple[int, int, int]:
        return self.grid.shape


def ct_to_attenuation(volume: ImagingVolume, *, energy_kev: float) -> ImagingVolume:
    """HU -> water-scaled attenuation ``max(1 + HU/1000, 0) * 0.02059`` mm^-1 (60 keV only).

    Evaluated in FP64 one slice at a time and rounded once to FP32.
    """
    if not isinstance(volume, ImagingVolume):
        raise ContractError("volume must be an ImagingVolume")
    if volume.metadata.value_units != "HU":
        raise ContractError("ct_to_attenuation requires volume units='HU'")
    if finite_scalar(energy_kev, "energy_kev", minimum=0.0) != 60.0:
        raise ContractError("the water-scaled HU model supports energy_kev=60.0 only")
    out = np.empty(volume.values.shape, dtype=np.float32)
    for z in range(out.shape[0]):
        out[z] = hu_to_mu(volume.values[z])
    return ImagingVolume(out, volume.grid,
                         replace(volume.metadata, value_units="mm^-1", measurement_unit_code=None))


def hu_to_mu(hu: np.ndarray) -> np.ndarray:
    """FP64 ``max(1 + HU/1000, 0) * 0.02059`` rounded once to FP32."""
    value = np.asarray(hu, dtype=np.float64) / 1000.0
    value += 1.0
    np.maximum(value, 0.0, out=value)
    value *= WATER_60KEV_MM
    return value.astype(np.float32)


def standard_views(
    grid: GridSpec,
    names: Sequence[str] = ("ap", "lateral", "oblique"),
    *,
    shape: tuple[int, int] = (512, 512),
) -> BatchedGeometry:
    """Centred AP (+Y source), lateral (+X) and oblique cone views covering the grid.

    With D the support diagonal: SOD = max(1000, 2D), SDD = max(1500, 3D), panel
    width 1.05 D SDD / (SOD - D/2), all mm.
    """
    if not isinstance(grid, GridSpec):
        raise ContractError("grid must be a GridSpec in RAS coordinates")
    if isinstance(names, str) or not names:
        raise ContractError("names must be a non-empty sequence of view names")
    angles = {"ap": math.pi, "lateral": math.pi / 2, "oblique": 3 * math.pi / 4}
    if any(name not in angles for name in names):
        raise ContractError("standard view names are ap, lateral and oblique")
    if len(shape) != 2 or any(type(n) is not int or n < 1 for n in shape):
        raise ContractError("shape must contain positive integer (rows,columns)")
    nz, ny, nx = grid.shape
    centre = grid.grid_to_object(((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2))
    diagonal = math.hypot(nx * grid.spacing_mm[0], ny * grid.spacing_mm[1], nz * grid.spacing_mm[2])
    sod, sdd = max(1000.0, 2.0 * diagonal), max(1500.0, 3.0 * diagonal)
    width = 1.05 * diagonal * sdd / (sod - diagonal / 2.0)
    if not math.isfinite(width):
        raise ContractError("grid extent exceeds the finite standard-view geometry range")
    intrinsics = ConeBeamIntrinsics(sod, sdd, shape, (width / shape[1], width / shape[0]), centre_mm=centre)
    return intrinsics.batch(tuple(angles[name] for name in names))
