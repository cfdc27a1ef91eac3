"""Sampled-grid metadata: shape, spacing, origin and orientation in millimetres.

``GridSpec`` keeps the reference field order and conventions
(hcltech-robotics/dpt ``python/dpt/volumes.py:17-93``): the sample buffer is
contiguous and x-fastest with ``shape = (nz, ny, nx)``, ``spacing_mm = (x, y, z)``,
``origin_mm`` is the object-frame position of sample ``(0, 0, 0)`` and
``orientation`` is a row-major rotation whose columns are the grid axes in
object coordinates.  The sampled field is extended by half a sample outside the
outer centres (clamped interpolation) and is zero beyond that support.
"""

from __future__ import annotations

from dataclasses import dataclass

from .contracts import ContractError
from .geometry import IDENTITY, Matrix3, Vector3, matvec, rotation_matrix, transpose, vector3


@dataclass(frozen=True, slots=True)
class GridSpec:
    """Oriented anisotropic sample grid; the origin is the first sample centre."""

    shape: tuple[int, int, int]
    spacing_mm: Vector3
    origin_mm: Vector3 = (0.0, 0.0, 0.0)
    orientation: Matrix3 = IDENTITY

    def __post_init__(self) -> None:
        if len(self.shape) != 3 or any(type(n) is not int or n < 1 for n in self.shape):
            raise ContractError("grid shape is (nz, ny, nx), each a positive integer")
        object.__setattr__(self, "shape", tuple(self.shape))
        object.__setattr__(self, "spacing_mm", vector3(self.spacing_mm, "spacing_mm"))
        object.__setattr__(self, "origin_mm", vector3(self.origin_mm, "origin_mm"))
        object.__setattr__(self, "orientation", rotation_matrix(self.orientation, "orientation"))
        if min(self.spacing_mm) <= 0.0:
            raise ContractError("grid spacing must be positive")
        if self.voxels > 2**31 - 1:
            raise ContractError("grid exceeds signed 32-bit indexing")

    @classmethod
    def from_axes(
        cls,
        *,
        nx: int,
        ny: int,
        nz: int,
        spacing_x_mm: float,
        spacing_y_mm: float,
        spacing_z_mm: float,
        origin_mm: Vector3 = (0.0, 0.0, 0.0),
        orientation: Matrix3 = IDENTITY,
    ) -> GridSpec:
        """Construct from named per-axis counts and spacings."""
        return cls((nz, ny, nx), (spacing_x_mm, spacing_y_mm, spacing_z_mm), origin_mm, orientation)

    @property
    def shape_zyx(self) -> tuple[int, int, int]:
        return self.shape

    @property
    def spacing_xyz_mm(self) -> Vector3:
        return self.spacing_mm

    @property
    def voxels(self) -> int:
        nz, ny, nx = self.shape
        return nz * ny * nx

    def object_to_grid(self, point_mm: Vector3) -> Vector3:
        """Continuous grid index ``(x, y, z)`` of an object-frame point."""
        offset = tuple(point_mm[i] - self.origin_mm[i] for i in range(3))
        aligned = matvec(transpose(self.orientation), offset)  # type: ignore[arg-type]
        return tuple(aligned[i] / self.spacing_mm[i] for i in range(3))  # type: ignore[return-value]

    def grid_to_object(self, index: Vector3) -> Vector3:
        """Object-frame position of a continuous grid index ``(x, y, z)``."""
        scaled = tuple(index[i] * self.spacing_mm[i] for i in range(3))
        aligned = matvec(self.orientation, scaled)  # type: ignore[arg-type]
        return tuple(aligned[i] + self.origin_mm[i] for i in range(3))  # type: ignore[return-value]

    @property
    def support(self) -> tuple[Vector3, Vector3]:
        nz, ny, nx = self.shape
        return (-0.5, -0.5, -0.5), (nx - 0.5, ny - 0.5, nz - 0.5)

    def object_to_grid_matrix(self) -> tuple[float, ...]:
        """Row-major ``M = diag(1/h) G^T``: grid index = M (x_object - origin).

        Entry ``M[i][j] = orientation[3*j + i] / spacing[i]``, each one IEEE
        division (reference ``python/dpt/projection.py:565-568``).
        """
        matrix = tuple(
            self.orientation[3 * j + i] / self.spacing_mm[i] for i in range(3) for j in range(3)
        )
        return matrix
