"""Analytic ellipsoids, sampled phantoms and circular cone scans for checks and benchmarks.

``Ellipsoid``, ``sample_ellipsoids`` and ``circular_cone_beam`` keep the
reference's contracts (hcltech-robotics/dpt ``python/dpt/phantoms.py:25-226``).
The seeded synthetic volumes (``ellipsoid_phantom``, ``chest_phantom``,
``head_phantom``) stand in for the scanned volumes of the reference's published
runs, which are not available here; they follow the described composition
(air / body / lungs / spine and ribs in HU for the chest, skull shell / brain /
ventricles for the head) and are converted to attenuation with the 60 keV water
model ``max(1 + HU/1000, 0) * 0.02059``.
"""

from __future__ import annotations

import math
from collections.abc import Iterable
from dataclasses import dataclass

import numpy as np

from .contracts import ContractError, finite_scalar
from .geometry import (
    IDENTITY,
    DetectorGeometry,
    Matrix3,
    Vector3,
    matvec,
    rotation_matrix,
    transpose,
    vector3,
)
from .imaging import hu_to_mu
from .volumes import GridSpec


@dataclass(frozen=True, slots=True)
class Ellipsoid:
    """``mu(x) = coefficient`` inside ``|R^T (x - c) / axes| <= 1`` (object mm, mm^-1)."""

    axes_mm: Vector3
    attenuation_mm_inverse: float
    centre_mm: Vector3 = (0.0, 0.0, 0.0)
    orientation: Matrix3 = IDENTITY

    def __post_init__(self) -> None:
        object.__setattr__(self, "axes_mm", vector3(self.axes_mm, "axes_mm"))
        if min(self.axes_mm) <= 0:
            raise ContractError("ellipsoid axes must be positive")
        object.__setattr__(self, "centre_mm", vector3(self.centre_mm, "centre_mm"))
        object.__setattr__(self, "orientation", rotation_matrix(self.orientation))
        object.__setattr__(
            self,
            "attenuation_mm_inverse",
            finite_scalar(self.attenuation_mm_inverse, "attenuation_mm_inverse", minimum=0),
        )

    def optical_depth(self, source_mm: Vector3, target_mm: Vector3) -> float:
        """Analytic ``coefficient * |segment inside the ellipsoid|`` (0 for misses)."""
        source, target = vector3(source_mm, "source_mm"), vector3(target_mm, "target_mm")
        rt = transpose(self.orientation)
        start = matvec(rt, tuple(source[i] - self.centre_mm[i] for i in range(3)))  # type: ignore[arg-type]
        delta = matvec(rt, tuple(target[i] - source[i] for i in range(3)))  # type: ignore[arg-type]
        # unit sphere coordinates
        o = [start[i] / self.axes_mm[i] for i in range(3)]
        d = [delta[i] / self.axes_mm[i] for i in range(3)]
        dd = math.fsum(x * x for x in d)
        if dd == 0.0:
            return 0.0
        # closest approach parameter and squared distance, relative to the chord midpoint
        t0 = -math.fsum(o[i] * d[i] for i in range(3)) / dd
        closest = [o[i] + t0 * d[i] for i in range(3)]
        h2 = 1.0 - math.fsum(x * x for x in closest)
        if not all(math.isfinite(x) for x in (t0, h2)):
            raise ContractError("ray exceeds the finite analytic ellipsoid range")
        if h2 <= 0.0:
            return 0.0
        half = math.sqrt(h2 / dd)
        lower, upper = max(t0 - half, 0.0), min(t0 + half, 1.0)
        length = max(0.0, upper - lower) * math.dist(source, target)
        return finite_scalar(self.attenuation_mm_inverse * length, "analytic optical depth")


def _object_coordinates(grid: GridSpec, z: int) -> list[np.ndarray]:
    nz, ny, nx = grid.shape
    x = np.arange(nx, dtype=np.float64)[None, :] * grid.spacing_mm[0]
    y = np.arange(ny, dtype=np.float64)[:, None] * grid.spacing_mm[1]
    zz = z * grid.spacing_mm[2]
    o = grid.orientation
    return [grid.origin_mm[a] + o[3 * a] * x + o[3 * a + 1] * y + o[3 * a + 2] * zz for a in range(3)]


def sample_ellipsoids(grid: GridSpec, ellipsoids: Iterable[Ellipsoid], *, dtype: str = "float32"):
    """``values[z,y,x] = sum_j mu_j(grid_to_object(x,y,z))`` (additive overlaps)."""
    if dtype not in ("float32", "float64"):
        raise ContractError("phantom dtype must be float32 or float64")
    models = tuple(ellipsoids)
    if any(not isinstance(m, Ellipsoid) for m in models):
        raise ContractError("supply Ellipsoid objects")
    out = np.zeros(grid.shape, dtype=dtype)
    for z in range(grid.shape[0]):
        coords = _object_coordinates(grid, z)
        for m in models:
            rt = transpose(m.orientation)
            r2 = np.zeros_like(coords[0])
            for a in range(3):
                local = sum(rt[3 * a + k] * (coords[k] - m.centre_mm[k]) for k in range(3))
                r2 += (local / m.axes_mm[a]) ** 2
            out[z] += (r2 <= 1.0) * m.attenuation_mm_inverse
    return out


def circular_cone_beam(
    angles_radians: Iterable[float],
    *,
    source_radius_mm: float,
    detector_radius_mm: float,
    shape_rows_columns: tuple[int, int],
    spacing_column_row_mm: tuple[float, float],
    centre_mm: Vector3 = (0.0, 0.0, 0.0),
) -> tuple[DetectorGeometry, ...]:
    """Source at ``centre + R_s (cos a, sin a, 0)``, flat panel centred at ``centre - R_d n``."""
    rs = finite_scalar(source_radius_mm, "source_radius_mm", minimum=0)
    rd = finite_scalar(detector_radius_mm, "detector_radius_mm", minimum=0)
    if rs == 0 or rd == 0:
        raise ContractError("source and detector radii must be positive")
    centre = vector3(centre_mm, "centre_mm")
    rows, columns = shape_rows_columns
    if any(type(n) is not int or n <= 0 for n in (rows, columns)):
        raise ContractError("shape_rows_columns needs positive integer rows and columns")
    pitch_c, pitch_r = (finite_scalar(x, "pixel spacing", minimum=0) for x in spacing_column_row_mm)
    if min(pitch_c, pitch_r) <= 0:
        raise ContractError("pixel spacing must be positive")
    panels = []
    for raw in angles_radians:
        a = finite_scalar(raw, "angle_radians")
        n = (math.cos(a), math.sin(a), 0.0)
        u = (-n[1], n[0], 0.0)
        v = (0.0, 0.0, 1.0)
        source = tuple(centre[k] + rs * n[k] for k in range(3))
        origin = tuple(
            centre[k] - rd * n[k] - 0.5 * (columns - 1) * pitch_c * u[k] - 0.5 * (rows - 1) * pitch_r * v[k]
            for k in range(3)
        )
        panels.append(DetectorGeometry(source, origin, u, v, (pitch_c, pitch_r), (rows, columns)))  # type: ignore[arg-type]
    return tuple(panels)


# --------------------------------------------------------------- synthetic scans


def centred_grid(shape: tuple[int, int, int], spacing_mm: Vector3, orientation: Matrix3 = IDENTITY) -> GridSpec:
    """Grid whose sample centres are centred on the object origin."""
    nz, ny, nx = shape
    half = ((nx - 1) / 2.0 * spacing_mm[0], (ny - 1) / 2.0 * spacing_mm[1], (nz - 1) / 2.0 * spacing_mm[2])
    offset = matvec(orientation, half)  # type: ignore[arg-type]
    return GridSpec(shape, spacing_mm, tuple(-x for x in offset), orientation)  # type: ignore[arg-type]


def random_rotation(rng: np.random.Generator) -> Matrix3:
    """Uniform random rotation (normalised quaternion)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    m = (
        1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y),
    )
    return tuple(float(v) for v in m)  # type: ignore[return-value]


def ellipsoid_phantom(grid: GridSpec, *, seed: int = 0, count: int = 6,
                      background: float = 0.002) -> tuple[np.ndarray, tuple[Ellipsoid, ...]]:
    """``count`` random ellipsoids (semi-axes 5-25 mm, random orientation, mu 0.01-0.05
    /mm, additive) on a ``background`` /mm field, centres inside the central half."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    extent = (nx * grid.spacing_mm[0], ny * grid.spacing_mm[1], nz * grid.spacing_mm[2])
    centre = grid.grid_to_object(((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2))
    models = []
    for _ in range(count):
        axes = tuple(float(a) for a in rng.uniform(5.0, 25.0, 3))
        offset = tuple(float(rng.uniform(-0.25, 0.25) * e) for e in extent)
        models.append(Ellipsoid(axes, float(rng.uniform(0.01, 0.05)),  # type: ignore[arg-type]
                                tuple(centre[k] + offset[k] for k in range(3)), random_rotation(rng)))  # type: ignore[arg-type]
    values = sample_ellipsoids(grid, models)
    values += np.float32(background)
    return values, tuple(models)


def _ellipse_mask(coords, centre, axes) -> np.ndarray:
    r2 = np.zeros_like(coords[0])
    for a in range(len(axes)):
        r2 = r2 + ((coords[a] - centre[a]) / axes[a]) ** 2
    return r2 <= 1.0


def chest_phantom(grid: GridSpec, *, seed: int = 0) -> np.ndarray:
    """Chest-like attenuation volume (FP32 mm^-1) in the grid's object frame.

    HU composition: air -1000 outside a body ellipse (0 HU +- 40 HU Gaussian
    noise), two lung ellipsoids (-850 HU), a spine cylinder along z (+1200 HU) and
    rib cylinders (+700 to +1100 HU); converted with the 60 keV water model.
    """
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    ex = nx * grid.spacing_mm[0]
    ey = ny * grid.spacing_mm[1]
    ez = nz * grid.spacing_mm[2]
    body_axes = (0.44 * ex, 0.32 * ey)
    lung_axes = (0.15 * ex, 0.2 * ey, 0.4 * ez)
    lungs = ((-0.2 * ex, -0.02 * ey, 0.0), (0.2 * ex, -0.02 * ey, 0.0))
    spine_centre, spine_radius = (0.0, 0.22 * ey), 0.06 * ex
    ribs = [(sign * 0.36 * ex, k * 0.06 * ey, 0.018 * ex, 700.0 + 100.0 * abs(k))
            for sign in (-1.0, 1.0) for k in range(-4, 5)]
    out = np.empty(grid.shape, dtype=np.float32)
    for z in range(nz):
        x, y, zz = _object_coordinates(grid, z)
        hu = np.full(x.shape, -1000.0)
        body = _ellipse_mask((x, y), (0.0, 0.0), body_axes)
        hu[body] = rng.normal(0.0, 40.0, int(body.sum()))
        for centre in lungs:
            hu[_ellipse_mask((x, y, zz), centre, lung_axes) & body] = -850.0
        hu[_ellipse_mask((x, y), spine_centre, (spine_radius, spine_radius))] = 1200.0
        for cx, cy, r, value in ribs:
            hu[_ellipse_mask((x, y), (cx, cy), (r, r)) & body] = value
        out[z] = hu_to_mu(hu)
    return out


def head_phantom(grid: GridSpec, *, seed: int = 0) -> np.ndarray:
    """Head-like attenuation volume in RAS object coordinates (x right, y anterior,
    z superior): a skull shell (+1000 HU; 6 mm, 10 mm over the occiput), brain
    30 +- 10 HU, two ventricles (5 HU), a calcified pineal spot (+400 HU, off the
    midline), two orbits (fat, -100 HU) and a frontal sinus (air) cut into the
    anterior skull, two petrous ridges (+1500 HU) and a mandible arc (+1800 HU)
    below; air outside; 60 keV water model, FP32 mm^-1.  The anterior and inferior
    structures break the shell's symmetries so that every rotation is observable
    from two orthogonal views."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = grid.shape
    centre = grid.grid_to_object(((nx - 1) / 2, (ny - 1) / 2, (nz - 1) / 2))
    extent = (nx * grid.spacing_mm[0], ny * grid.spacing_mm[1], nz * grid.spacing_mm[2])
    ex, ey, ez = extent
    outer = (0.42 * ex, 0.46 * ey, 0.46 * ez)
    inner = tuple(a - 6.0 for a in outer)
    occiput = (0.0, -0.10 * ey, 0.0)
    occiput_axes = (outer[0] - 10.0, outer[1] - 4.0, outer[2] - 10.0)
    ventricles = ((-0.06 * ex, 0.0, 0.0), (0.06 * ex, 0.0, 0.0))
    ventricle_axes = (0.04 * ex, 0.12 * ey, 0.15 * ez)
    pineal = ((0.03 * ex, -0.08 * ey, 0.05 * ez), (0.015 * ex, 0.015 * ey, 0.02 * ez))
    orbits = (((-0.13 * ex, 0.38 * ey, -0.08 * ez), (0.07 * ex, 0.08 * ey, 0.09 * ez)),
              ((0.13 * ex, 0.38 * ey, -0.08 * ez), (0.07 * ex, 0.08 * ey, 0.09 * ez)))
    sinus = ((0.01 * ex, 0.40 * ey, 0.12 * ez), (0.10 * ex, 0.05 * ey, 0.07 * ez))
    petrous = (((-0.22 * ex, -0.05 * ey, -0.25 * ez), (0.14 * ex, 0.03 * ey, 0.04 * ez)),
               ((0.22 * ex, -0.05 * ey, -0.25 * ez), (0.14 * ex, 0.03 * ey, 0.04 * ez)))
    jaw_outer = ((0.0, 0.22 * ey, -0.40 * ez), (0.30 * ex, 0.22 * ey, 0.06 * ez))
    jaw_inner = ((0.0, 0.16 * ey, -0.40 * ez), (0.25 * ex, 0.18 * ey, 0.07 * ez))
    out = np.empty(grid.shape, dtype=np.float32)
    for z in range(nz):
        coords = [c - centre[k] for k, c in enumerate(_object_coordinates(grid, z))]
        hu = np.full(coords[0].shape, -1000.0)
        skull = _ellipse_mask(coords, (0.0, 0.0, 0.0), outer)
        brain = _ellipse_mask(coords, (0.0, 0.0, 0.0), inner) & _ellipse_mask(coords, occiput, occiput_axes)
        hu[skull] = 1000.0
        hu[brain] = rng.normal(30.0, 10.0, int(brain.sum()))
        for c in ventricles:
            hu[_ellipse_mask(coords, c, ventricle_axes) & brain] = 5.0
        hu[_ellipse_mask(coords, *pineal) & brain] = 400.0
        for c, axes in orbits:
            hu[_ellipse_mask(coords, c, axes)] = -100.0
        hu[_ellipse_mask(coords, *sinus)] = -1000.0
        for c, axes in petrous:
            hu[_ellipse_mask(coords, c, axes)] = 1500.0
        hu[_ellipse_mask(coords, *jaw_outer) & ~_ellipse_mask(coords, *jaw_inner)] = 1800.0
        out[z] = hu_to_mu(hu)
    return out
