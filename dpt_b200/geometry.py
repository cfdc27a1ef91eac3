"""Rigid geometry in millimetres: poses, detector panels, ray bundles, cone-beam scans.

The objects keep the reference's constructor signatures, field orders and
conventions (hcltech-robotics/dpt ``python/dpt/geometry.py``) so code written
against the reference builds the same acquisitions here:

* rotations are row-major 3x3 tuples acting on column vectors; a packed pose is
  the 9 rotation entries followed by the translation (12 doubles), mapping object
  points into world coordinates (``RigidTransform``, reference ``:66-97``);
* a flat panel (``DetectorGeometry``, ``:100-221``) has ``shape = (rows, columns)``,
  ``spacing_mm = (column pitch, row pitch)`` and ``origin_mm`` at pixel (0, 0);
  ``u`` advances columns and ``v`` advances rows;
* ``ParallelGeometry`` (``:320-372``) and ``CurvedDetectorGeometry`` (``:382-436``)
  describe finite parallel segments and cylindrical panels;
* ``BatchedGeometry`` (``:461-614``) stacks equally shaped panels into a
  ``(views, rows, columns)`` image; ``ConeBeamIntrinsics`` (``:617-701``) builds
  circular cone scans;
* ``compose_pose`` / ``right_jacobian_se3`` / ``chart_gradient`` (``:742-846``)
  implement the SE(3) chart ``anchor @ exp(xi^)`` with ``xi = (t, omega)``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from itertools import pairwise
from typing import Literal

from .contracts import ContractError, finite_tuple

Vector3 = tuple[float, float, float]
Matrix3 = tuple[float, float, float, float, float, float, float, float, float]
IDENTITY: Matrix3 = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)

# ------------------------------------------------------------------ algebra


def vector3(value: Vector3, name: str) -> Vector3:
    """Validate a 3-tuple of finite reals (any sign)."""
    return finite_tuple(value, name, minimum=None, length=3)  # type: ignore[return-value]


def dot(a: Vector3, b: Vector3) -> float:
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def cross(a: Vector3, b: Vector3) -> Vector3:
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def matvec(m: Matrix3, v: Vector3) -> Vector3:
    return (
        m[0] * v[0] + m[1] * v[1] + m[2] * v[2],
        m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
        m[6] * v[0] + m[7] * v[1] + m[8] * v[2],
    )


def transpose(m: Matrix3) -> Matrix3:
    return (m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8])


def matmul(a: Matrix3, b: Matrix3) -> Matrix3:
    return tuple(  # type: ignore[return-value]
        a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j]
        for i in range(3)
        for j in range(3)
    )


def rotation_matrix(value: Matrix3, name: str = "rotation") -> Matrix3:
    """Validate an orthonormal (to 1e-10), right-handed row-major rotation."""
    value = finite_tuple(value, name, minimum=None, length=9)  # type: ignore[assignment]
    gram = matmul(transpose(value), value)
    if max(abs(g - e) for g, e in zip(gram, IDENTITY, strict=True)) > 1e-10:
        raise ContractError(f"{name} must be orthonormal to 1e-10")
    c0 = (value[0], value[3], value[6])
    c1 = (value[1], value[4], value[7])
    c2 = (value[2], value[5], value[8])
    if dot(cross(c0, c1), c2) < 0.0:
        raise ContractError(f"{name} must be right-handed")
    return tuple(float(x) for x in value)  # type: ignore[return-value]


def _add(a: Vector3, b: Vector3) -> Vector3:
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _sub(a: Vector3, b: Vector3) -> Vector3:
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _scale(s: float, a: Vector3) -> Vector3:
    return (s * a[0], s * a[1], s * a[2])


# ---------------------------------------------------------------- transforms


@dataclass(frozen=True, slots=True)
class RigidTransform:
    """Object-to-world map ``x_world = R x_object + t`` (t in mm)."""

    rotation: Matrix3 = IDENTITY
    translation_mm: Vector3 = (0.0, 0.0, 0.0)

    def __post_init__(self) -> None:
        object.__setattr__(self, "rotation", rotation_matrix(self.rotation))
        object.__setattr__(self, "translation_mm", vector3(self.translation_mm, "translation"))

    def point(self, point_mm: Vector3) -> Vector3:
        return _add(matvec(self.rotation, point_mm), self.translation_mm)

    def direction(self, direction: Vector3) -> Vector3:
        return matvec(self.rotation, direction)

    def inverse(self) -> RigidTransform:
        rt = transpose(self.rotation)
        return RigidTransform(rt, _scale(-1.0, matvec(rt, self.translation_mm)))

    def compose(self, right: RigidTransform) -> RigidTransform:
        """``self @ right`` (``right`` is applied first)."""
        return RigidTransform(matmul(self.rotation, right.rotation), self.point(right.translation_mm))

    def packed(self) -> tuple[float, ...]:
        """Twelve doubles: row-major rotation, then translation."""
        return (*self.rotation, *self.translation_mm)


# -------------------------------------------------------------------- panels


def _panel_shape(shape: tuple[int, int]) -> None:
    if (
        not isinstance(shape, tuple)
        or len(shape) != 2
        or any(type(n) is not int or n <= 0 for n in shape)
    ):
        raise ContractError("detector shape must be (rows,columns), both positive integers")
    if shape[0] * shape[1] > 2**31 - 1:
        raise ContractError("detector exceeds signed 32-bit indexing")


def _pixel_index(row: int, column: int, shape: tuple[int, int]) -> None:
    if type(row) is not int or type(column) is not int:
        raise ContractError("pixel indices must be integers")
    if not (0 <= row < shape[0] and 0 <= column < shape[1]):
        raise ContractError("pixel index outside detector")


def _flat_pixel(origin: Vector3, u: Vector3, v: Vector3, spacing: tuple[float, float],
                row: int, column: int) -> Vector3:
    return tuple(  # type: ignore[return-value]
        origin[i] + column * spacing[0] * u[i] + row * spacing[1] * v[i] for i in range(3)
    )


@dataclass(frozen=True, slots=True)
class DetectorGeometry:
    """Flat panel of finite source-to-pixel segments (cone beam).

    ``shape = (rows, columns)``, ``spacing_mm = (column pitch, row pitch)``;
    ``u`` and ``v`` are perpendicular unit vectors along columns and rows.
    """

    source_mm: Vector3
    origin_mm: Vector3
    u: Vector3
    v: Vector3
    spacing_mm: tuple[float, float]
    shape: tuple[int, int]

    def __post_init__(self) -> None:
        for name in ("source_mm", "origin_mm", "u", "v"):
            object.__setattr__(self, name, vector3(getattr(self, name), name))
        if abs(dot(self.u, self.u) - 1.0) > 1e-10 or abs(dot(self.v, self.v) - 1.0) > 1e-10:
            raise ContractError("detector basis vectors must have unit length")
        if abs(dot(self.u, self.v)) > 1e-10:
            raise ContractError("detector basis vectors must be perpendicular")
        spacing = finite_tuple(self.spacing_mm, "pixel spacing", positive=True, length=2)
        if (
            not isinstance(self.shape, tuple)
            or len(self.shape) != 2
            or any(type(n) is not int or n <= 0 for n in self.shape)
        ):
            raise ContractError("detector shape is (height, width), both positive integers")
        object.__setattr__(self, "spacing_mm", spacing)
        offset = _sub(self.source_mm, self.origin_mm)
        if abs(dot(offset, cross(self.u, self.v))) <= 1e-12:
            raise ContractError("source must lie outside the detector plane")
        if self.pixels > 2**31 - 1:
            raise ContractError("detector exceeds signed 32-bit indexing")

    @classmethod
    def from_axes(
        cls,
        *,
        source_mm: Vector3,
        origin_mm: Vector3,
        u: Vector3,
        v: Vector3,
        rows: int,
        columns: int,
        spacing_column_mm: float,
        spacing_row_mm: float,
    ) -> DetectorGeometry:
        return cls(source_mm, origin_mm, u, v, (spacing_column_mm, spacing_row_mm), (rows, columns))

    @property
    def shape_rows_columns(self) -> tuple[int, int]:
        return self.shape

    @property
    def spacing_columns_rows_mm(self) -> tuple[float, float]:
        return self.spacing_mm

    @property
    def pixels(self) -> int:
        return self.shape[0] * self.shape[1]

    def pixel_centre(self, row: int, column: int) -> Vector3:
        _pixel_index(row, column, self.shape)
        return _flat_pixel(self.origin_mm, self.u, self.v, self.spacing_mm, row, column)

    def projection_matrix(self) -> tuple[tuple[float, float, float, float], ...]:
        """3x4 map of homogeneous world points to ``[column, row, depth]``."""
        normal = cross(self.u, self.v)
        offset = _sub(self.origin_mm, self.source_mm)
        distance = dot(normal, offset)
        rows = []
        for axis, pitch in zip((self.u, self.v), self.spacing_mm, strict=True):
            along = dot(axis, offset)
            coefficient = tuple((distance * axis[i] - along * normal[i]) / pitch for i in range(3))
            rows.append((*coefficient, -dot(coefficient, self.source_mm)))  # type: ignore[arg-type]
        rows.append((*normal, -dot(normal, self.source_mm)))
        return tuple(rows)  # type: ignore[return-value]

    def project_point(self, point_mm: Vector3) -> tuple[float, float]:
        """Continuous ``(row, column)`` where the source-to-point line meets the panel."""
        p = (*vector3(point_mm, "point_mm"), 1.0)
        h = [sum(a * b for a, b in zip(row, p, strict=True)) for row in self.projection_matrix()]
        if abs(h[2]) <= 1e-12:
            raise ContractError("source-to-point line is parallel to the detector plane")
        return h[1] / h[2], h[0] / h[2]


@dataclass(frozen=True, slots=True)
class RayBundleGeometry:
    """Explicit finite world segments; ``view_offsets`` partitions them into views."""

    sources_mm: tuple[Vector3, ...]
    endpoints_mm: tuple[Vector3, ...]
    view_offsets: tuple[int, ...] | None = None

    def __post_init__(self) -> None:
        if (
            not isinstance(self.sources_mm, tuple)
            or not isinstance(self.endpoints_mm, tuple)
            or not self.sources_mm
            or len(self.sources_mm) != len(self.endpoints_mm)
        ):
            raise ContractError("ray sources/endpoints must be equal non-empty immutable tuples")
        sources = tuple(vector3(s, "ray source") for s in self.sources_mm)
        endpoints = tuple(vector3(e, "ray endpoint") for e in self.endpoints_mm)
        for s, e in zip(sources, endpoints, strict=True):
            if s == e or not math.isfinite(math.dist(s, e)):
                raise ContractError("ray segments must have finite positive length")
        if len(sources) > 2**31 - 1:
            raise ContractError("ray bundle exceeds signed 32-bit indexing")
        offsets = self.view_offsets if self.view_offsets is not None else (0, len(sources))
        if (
            not isinstance(offsets, tuple)
            or len(offsets) < 2
            or any(type(o) is not int for o in offsets)
            or offsets[0] != 0
            or offsets[-1] != len(sources)
            or any(a >= b for a, b in pairwise(offsets))
        ):
            raise ContractError("view_offsets must partition the bundle into non-empty views")
        object.__setattr__(self, "sources_mm", sources)
        object.__setattr__(self, "endpoints_mm", endpoints)
        object.__setattr__(self, "view_offsets", offsets)

    @classmethod
    def from_views(cls, views: tuple[DetectorGeometry, ...]) -> RayBundleGeometry:
        """Flatten flat panels in view, row, column order."""
        if (
            not isinstance(views, tuple)
            or not views
            or any(not isinstance(v, DetectorGeometry) for v in views)
        ):
            raise ContractError("ray bundle views must be a non-empty tuple of DetectorGeometry")
        sources: list[Vector3] = []
        endpoints: list[Vector3] = []
        offsets = [0]
        for panel in views:
            for row in range(panel.shape[0]):
                for column in range(panel.shape[1]):
                    sources.append(panel.source_mm)
                    endpoints.append(panel.pixel_centre(row, column))
            offsets.append(len(sources))
        return cls(tuple(sources), tuple(endpoints), tuple(offsets))

    @property
    def pixels(self) -> int:
        return len(self.sources_mm)

    @property
    def rays(self) -> int:
        return self.pixels

    def segment(self, ray: int) -> tuple[Vector3, Vector3]:
        if type(ray) is not int or not 0 <= ray < self.pixels:
            raise ContractError("ray index must be an integer inside the bundle")
        return self.sources_mm[ray], self.endpoints_mm[ray]


@dataclass(frozen=True, slots=True)
class ParallelGeometry:
    """Finite parallel segments ``source = endpoint - length_mm * direction``."""

    origin_mm: Vector3
    direction: Vector3
    length_mm: float
    u: Vector3
    v: Vector3
    spacing_mm: tuple[float, float]
    shape: tuple[int, int]

    def __post_init__(self) -> None:
        direction = vector3(self.direction, "parallel direction")
        if abs(dot(direction, direction) - 1.0) > 1e-10:
            raise ContractError("parallel direction must have unit length")
        length = finite_tuple((self.length_mm,), "parallel length", positive=True)[0]
        origin = vector3(self.origin_mm, "parallel origin")
        source = _sub(origin, _scale(length, direction))
        panel = DetectorGeometry(source, origin, self.u, self.v, self.spacing_mm, self.shape)
        object.__setattr__(self, "origin_mm", origin)
        object.__setattr__(self, "direction", direction)
        object.__setattr__(self, "length_mm", length)
        for name in ("u", "v", "spacing_mm", "shape"):
            object.__setattr__(self, name, getattr(panel, name))

    @property
    def pixels(self) -> int:
        return self.shape[0] * self.shape[1]

    def pixel_centre(self, row: int, column: int) -> Vector3:
        _pixel_index(row, column, self.shape)
        return _flat_pixel(self.origin_mm, self.u, self.v, self.spacing_mm, row, column)

    def segment(self, row: int, column: int) -> tuple[Vector3, Vector3]:
        end = self.pixel_centre(row, column)
        return _sub(end, _scale(self.length_mm, self.direction)), end


@dataclass(frozen=True, slots=True)
class CurvedDetectorGeometry:
    """Cylindrical panel around the axis through ``source_mm`` along ``v``.

    Column ``c`` lies at arc length ``c * spacing_mm[0]`` from pixel (0, 0):
    ``p = origin + (cos a - 1) radial + sin a * R * u + row * spacing_mm[1] * v``
    with ``a = c * spacing_mm[0] / R``.
    """

    source_mm: Vector3
    origin_mm: Vector3
    u: Vector3
    v: Vector3
    spacing_mm: tuple[float, float]
    shape: tuple[int, int]

    def __post_init__(self) -> None:
        panel = DetectorGeometry(
            self.source_mm, self.origin_mm, self.u, self.v, self.spacing_mm, self.shape
        )
        for name in ("source_mm", "origin_mm", "u", "v", "spacing_mm", "shape"):
            object.__setattr__(self, name, getattr(panel, name))
        radius = self.radius_mm
        if not math.isfinite(radius) or radius <= 0.0:
            raise ContractError("curved detector radius must be finite and positive")
        if abs(dot(self.radial_mm, self.u)) > 1e-10 * radius:
            raise ContractError("curved detector u must be tangent to its source-centred cylinder")
        if self.spacing_mm[0] * (self.shape[1] - 1) >= 2 * math.pi * radius:
            raise ContractError("curved detector columns must cover less than one full revolution")

    @property
    def radial_mm(self) -> Vector3:
        offset = _sub(self.origin_mm, self.source_mm)
        return _sub(offset, _scale(dot(offset, self.v), self.v))

    @property
    def radius_mm(self) -> float:
        r = self.radial_mm
        return math.sqrt(dot(r, r))

    @property
    def pixels(self) -> int:
        return self.shape[0] * self.shape[1]

    def pixel_centre(self, row: int, column: int) -> Vector3:
        _pixel_index(row, column, self.shape)
        radial, radius = self.radial_mm, self.radius_mm
        angle = column * self.spacing_mm[0] / radius
        c, s = math.cos(angle) - 1.0, math.sin(angle) * radius
        return tuple(  # type: ignore[return-value]
            self.origin_mm[i] + c * radial[i] + s * self.u[i] + row * self.spacing_mm[1] * self.v[i]
            for i in range(3)
        )


PanelGeometry = DetectorGeometry | ParallelGeometry | CurvedDetectorGeometry
AstraVector = tuple[float, ...]


@dataclass(frozen=True, slots=True)
class AstraVectorGeometry:
    """ASTRA ``cone_vec`` / ``parallel3d_vec`` rows ``(source|direction, centre, u, v)``."""

    kind: Literal["cone_vec", "parallel3d_vec"]
    shape_rows_columns: tuple[int, int]
    vectors: tuple[AstraVector, ...]

    def __post_init__(self) -> None:
        if self.kind not in ("cone_vec", "parallel3d_vec"):
            raise ContractError("ASTRA kind must be cone_vec or parallel3d_vec")
        _panel_shape(self.shape_rows_columns)
        if not isinstance(self.vectors, tuple) or not self.vectors:
            raise ContractError("ASTRA vectors must be a non-empty immutable tuple")
        object.__setattr__(
            self,
            "vectors",
            tuple(finite_tuple(row, "ASTRA vector", minimum=None, length=12) for row in self.vectors),
        )


@dataclass(frozen=True, slots=True)
class BatchedGeometry:
    """Equally shaped panels forming a ``(views, rows, columns)`` image."""

    views: tuple[PanelGeometry, ...]

    def __post_init__(self) -> None:
        kinds = (DetectorGeometry, ParallelGeometry, CurvedDetectorGeometry)
        if (
            not isinstance(self.views, tuple)
            or not self.views
            or any(not isinstance(view, kinds) for view in self.views)
        ):
            raise ContractError("views must be a non-empty immutable tuple of panel geometries")
        if any(view.shape != self.views[0].shape for view in self.views):
            raise ContractError("batched views must share (rows,columns)")
        if self.pixels > 2**31 - 1:
            raise ContractError("batched geometry exceeds signed 32-bit indexing")

    @property
    def shape_rows_columns(self) -> tuple[int, int]:
        return self.views[0].shape

    @property
    def shape(self) -> tuple[int, int, int]:
        return (len(self.views), *self.shape_rows_columns)

    @property
    def pixels(self) -> int:
        return len(self.views) * self.views[0].pixels

    @property
    def view_offsets(self) -> tuple[int, ...]:
        count = self.views[0].pixels
        return tuple(k * count for k in range(len(self.views) + 1))

    def segment(self, view: int, row: int, column: int) -> tuple[Vector3, Vector3]:
        if type(view) is not int or not 0 <= view < len(self.views):
            raise ContractError("view index must be inside the batch")
        panel = self.views[view]
        if isinstance(panel, ParallelGeometry):
            return panel.segment(row, column)
        return panel.source_mm, panel.pixel_centre(row, column)

    def to_astra_vectors(self) -> AstraVectorGeometry:
        """Export flat cone or parallel panels as ASTRA vectors (panel centre convention)."""
        parallel = isinstance(self.views[0], ParallelGeometry)
        for view in self.views:
            if isinstance(view, CurvedDetectorGeometry) or isinstance(view, ParallelGeometry) != parallel:
                raise ContractError(
                    "ASTRA vector export requires uniformly flat cone or parallel views"
                )
        rows, columns = self.shape_rows_columns
        vectors = []
        for view in self.views:
            du = _scale(view.spacing_mm[0], view.u)
            dv = _scale(view.spacing_mm[1], view.v)
            centre = tuple(
                view.origin_mm[i] + 0.5 * (columns - 1) * du[i] + 0.5 * (rows - 1) * dv[i]
                for i in range(3)
            )
            first = view.direction if isinstance(view, ParallelGeometry) else view.source_mm
            vectors.append((*first, *centre, *du, *dv))
        return AstraVectorGeometry(
            "parallel3d_vec" if parallel else "cone_vec", self.shape_rows_columns, tuple(vectors)
        )

    @classmethod
    def from_astra_vectors(
        cls,
        geometry: AstraVectorGeometry,
        *,
        length_scale_mm: float = 1.0,
        parallel_length_mm: float | None = None,
    ) -> BatchedGeometry:
        """Import ASTRA rows, scaling coordinates by ``length_scale_mm``."""
        scale = finite_tuple((length_scale_mm,), "length scale", positive=True)[0]
        if geometry.kind not in ("cone_vec", "parallel3d_vec"):
            raise ContractError("ASTRA kind must be cone_vec or parallel3d_vec")
        if geometry.kind == "parallel3d_vec" and parallel_length_mm is None:
            raise ContractError("parallel ASTRA import requires parallel_length_mm")
        rows, columns = geometry.shape_rows_columns
        views: list[PanelGeometry] = []
        for raw in geometry.vectors:
            values = finite_tuple(raw, "ASTRA vector", minimum=None, length=12)
            centre = tuple(scale * x for x in values[3:6])
            du_raw = tuple(scale * x for x in values[6:9])
            dv_raw = tuple(scale * x for x in values[9:12])
            du, dv = math.sqrt(dot(du_raw, du_raw)), math.sqrt(dot(dv_raw, dv_raw))  # type: ignore[arg-type]
            if min(du, dv) <= 0.0:
                raise ContractError("ASTRA pixel vectors must have positive length")
            u = tuple(x / du for x in du_raw)
            v = tuple(x / dv for x in dv_raw)
            origin = tuple(
                centre[i] - 0.5 * (columns - 1) * du_raw[i] - 0.5 * (rows - 1) * dv_raw[i]
                for i in range(3)
            )
            first = tuple(values[:3])
            if geometry.kind == "cone_vec":
                views.append(
                    DetectorGeometry(
                        tuple(scale * x for x in first), origin, u, v, (du, dv), (rows, columns)  # type: ignore[arg-type]
                    )
                )
            else:
                norm = math.sqrt(dot(first, first))  # type: ignore[arg-type]
                if norm <= 0.0:
                    raise ContractError("ASTRA parallel direction must have positive length")
                views.append(
                    ParallelGeometry(
                        origin,  # type: ignore[arg-type]
                        tuple(x / norm for x in first),  # type: ignore[arg-type]
                        float(parallel_length_mm),  # type: ignore[arg-type]
                        u,  # type: ignore[arg-type]
                        v,  # type: ignore[arg-type]
                        (du, dv),
                        (rows, columns),
                    )
                )
        return cls(tuple(views))


@dataclass(frozen=True, slots=True)
class ConeBeamIntrinsics:
    """Circular cone scan: source at ``(0, -SOD, 0)`` before a rotation about world z.

    The detector centre is ``(offset_column, SDD - SOD, offset_row)`` in the
    rotating frame, columns along +x and rows along +z; ``view(angle)`` rotates the
    frame by ``angle`` about z and translates it to ``centre_mm``.
    """

    source_object_distance_mm: float
    source_detector_distance_mm: float
    shape: tuple[int, int]
    spacing_mm: tuple[float, float]
    detector_offset_mm: tuple[float, float] = (0.0, 0.0)
    centre_mm: Vector3 = (0.0, 0.0, 0.0)

    def __post_init__(self) -> None:
        _panel_shape(self.shape)
        sod, sdd = finite_tuple(
            (self.source_object_distance_mm, self.source_detector_distance_mm),
            "SOD/SDD",
            positive=True,
            length=2,
        )
        if sdd <= sod:
            raise ContractError("source-detector distance must exceed source-object distance")
        object.__setattr__(self, "source_object_distance_mm", sod)
        object.__setattr__(self, "source_detector_distance_mm", sdd)
        object.__setattr__(
            self, "spacing_mm", finite_tuple(self.spacing_mm, "pixel spacing", positive=True, length=2)
        )
        object.__setattr__(
            self,
            "detector_offset_mm",
            finite_tuple(self.detector_offset_mm, "detector offset", minimum=None, length=2),
        )
        object.__setattr__(self, "centre_mm", vector3(self.centre_mm, "centre_mm"))
        self.view(0.0)

    def view(self, angle_rad: float) -> DetectorGeometry:
        angle = finite_tuple((angle_rad,), "view angle", minimum=None)[0]
        c, s = math.cos(angle), math.sin(angle)
        frame = RigidTransform((c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0), self.centre_mm)
        rows, columns = self.shape
        pitch_c, pitch_r = self.spacing_mm
        corner = (
            self.detector_offset_mm[0] - 0.5 * (columns - 1) * pitch_c,
            self.source_detector_distance_mm - self.source_object_distance_mm,
            self.detector_offset_mm[1] - 0.5 * (rows - 1) * pitch_r,
        )
        return DetectorGeometry(
            frame.point((0.0, -self.source_object_distance_mm, 0.0)),
            frame.point(corner),
            frame.direction((1.0, 0.0, 0.0)),
            frame.direction((0.0, 0.0, 1.0)),
            self.spacing_mm,
            self.shape,
        )

    def batch(self, angles_rad: tuple[float, ...]) -> BatchedGeometry:
        angles = finite_tuple(angles_rad, "angles", minimum=None)
        return BatchedGeometry(tuple(self.view(a) for a in angles))

    def ray_derivatives(self, angle_rad: float) -> tuple[tuple[Vector3, Vector3], ...]:
        """``(d source, d endpoint)`` for SOD, SDD, column offset and row offset."""
        angle = finite_tuple((angle_rad,), "view angle", minimum=None)[0]
        x = (math.cos(angle), math.sin(angle), 0.0)
        y = (-math.sin(angle), math.cos(angle), 0.0)
        minus_y = (-y[0], -y[1], -y[2])
        zero = (0.0, 0.0, 0.0)
        return ((minus_y, minus_y), (zero, y), (zero, x), (zero, (0.0, 0.0, 1.0)))


# ------------------------------------------------------------------ SE(3) chart


def _skew(w: Vector3) -> Matrix3:
    return (0.0, -w[2], w[1], w[2], 0.0, -w[0], -w[1], w[0], 0.0)


def _se3_coefficients(theta2: float) -> tuple[float, float, float, float, float]:
    """``A = sin t / t``, ``B = (1 - cos t)/t^2``, ``C = (t - sin t)/t^3`` and the
    derivatives ``dB/d(t^2)``, ``dC/d(t^2)`` as functions of ``t^2``.

    Near zero each is summed from its Taylor series in ``t^2`` (terms up to t^10,
    well below FP64 rounding for t^2 < 1e-2), avoiding the cancellation of the
    closed forms.
    """
    if not math.isfinite(theta2):
        raise ContractError("rotation norm exceeds the finite geometry range")
    if theta2 < 1e-2:
        # sum_k (-1)^k x^k / (2k+a)!  for a = 1 (A), 2 (B), 3 (C)
        def series(offset: int) -> float:
            total, term = 0.0, 1.0 / math.factorial(offset)
            for k in range(6):
                total += term
                term *= -theta2 / ((2 * k + offset + 1) * (2 * k + offset + 2))
            return total

        def derivative(offset: int) -> float:
            # d/dx sum_k (-1)^k x^k / (2k+offset)! = sum_{k>=1} (-1)^k k x^(k-1) / (2k+offset)!
            total, power = 0.0, 1.0
            for k in range(1, 7):
                total += (-1) ** k * k * power / math.factorial(2 * k + offset)
                power *= theta2
            return total

        return series(1), series(2), series(3), derivative(2), derivative(3)
    t = math.sqrt(theta2)
    s, c = math.sin(t), math.cos(t)
    a = s / t
    b = (1.0 - c) / theta2
    cc = (t - s) / (theta2 * t)
    # dB/d(t^2) = (dB/dt) / (2t), dC/d(t^2) = (dC/dt) / (2t)
    db = (t * s - 2.0 * (1.0 - c)) / (2.0 * theta2 * theta2)
    dc = (3.0 * s - t * (2.0 + c)) / (2.0 * theta2 * theta2 * t)
    return a, b, cc, db, dc


def _exp_se3(increment: tuple[float, ...]) -> tuple[Matrix3, Vector3]:
    rho = (increment[0], increment[1], increment[2])
    omega = (increment[3], increment[4], increment[5])
    k = _skew(omega)
    k2 = matmul(k, k)
    a, b, c, _, _ = _se3_coefficients(dot(omega, omega))
    rotation = tuple(IDENTITY[i] + a * k[i] + b * k2[i] for i in range(9))
    left = tuple(IDENTITY[i] + b * k[i] + c * k2[i] for i in range(9))
    return rotation, matvec(left, rho)  # type: ignore[arg-type, return-value]


def compose_pose(anchor: RigidTransform, increment: tuple[float, ...]) -> RigidTransform:
    """``anchor @ exp(xi^)`` for ``xi = (tx, ty, tz, rx, ry, rz)`` (mm, rad), acting on the right."""
    increment = finite_tuple(increment, "pose increment", minimum=None, length=6)
    rotation, translation = _exp_se3(increment)
    return anchor.compose(RigidTransform(rotation, translation))


def right_jacobian_se3(increment: tuple[float, ...]) -> tuple[tuple[float, ...], ...]:
    """``J_r(xi)`` with ``exp((xi + d)^) ~ exp(xi^) exp((J_r d)^)``, shape (6, 6).

    Rows are local-right coordinates at ``exp(xi^)``, columns additive chart
    coordinates.  Translation block ``R^T V``, rotation block ``I - B K + C K^2``
    and coupling ``R^T (dV/d omega_j) rho``.
    """
    increment = finite_tuple(increment, "pose increment", minimum=None, length=6)
    rho = (increment[0], increment[1], increment[2])
    omega = (increment[3], increment[4], increment[5])
    k = _skew(omega)
    k2 = matmul(k, k)
    a, b, c, db, dc = _se3_coefficients(dot(omega, omega))
    rotation = tuple(IDENTITY[i] + a * k[i] + b * k2[i] for i in range(9))
    rt = transpose(rotation)  # type: ignore[arg-type]
    left = tuple(IDENTITY[i] + b * k[i] + c * k2[i] for i in range(9))
    translation_block = matmul(rt, left)  # type: ignore[arg-type]
    rotation_block = tuple(IDENTITY[i] - b * k[i] + c * k2[i] for i in range(9))
    coupling = []
    for axis in range(3):
        e = _skew(tuple(1.0 if j == axis else 0.0 for j in range(3)))  # type: ignore[arg-type]
        ek, ke = matmul(e, k), matmul(k, e)
        # dV/d omega_axis, using d(theta^2)/d omega_axis = 2 omega_axis
        dv = tuple(
            2.0 * omega[axis] * (db * k[i] + dc * k2[i]) + b * e[i] + c * (ek[i] + ke[i])
            for i in range(9)
        )
        coupling.append(matvec(rt, matvec(dv, rho)))  # type: ignore[arg-type]
    jacobian = []
    for i in range(6):
        row = []
        for j in range(6):
            if i < 3 and j < 3:
                row.append(translation_block[3 * i + j])
            elif i < 3:
                row.append(coupling[j - 3][i])
            elif j >= 3:
                row.append(rotation_block[3 * (i - 3) + (j - 3)])
            else:
                row.append(0.0)
        jacobian.append(tuple(row))
    return tuple(jacobian)


def chart_gradient(
    increment: tuple[float, ...], right_gradient: tuple[float, ...]
) -> tuple[float, ...]:
    """``J_r(xi)^T g_right``: a local-right gradient in additive chart coordinates."""
    right_gradient = finite_tuple(right_gradient, "right tangent gradient", minimum=None, length=6)
    jacobian = right_jacobian_se3(increment)
    return tuple(sum(jacobian[i][j] * right_gradient[i] for i in range(6)) for j in range(6))
