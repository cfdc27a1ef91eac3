"""Host-side ray plans: geometry objects -> the flat FP64 tables the kernels read.

A plan holds, for one grid and one acquisition, everything that crosses the C
ABI apart from the field and poses: the ``dpt_problem`` scalars, the object-to-
grid map and either a per-view panel table (``DPT_VIEW_WORDS`` doubles per view)
or explicit source/endpoint arrays.

Panel records follow the reference's preparation (hcltech-robotics/dpt
``python/dpt/projection.py:561-591`` for flat cone panels, where the column and
row steps ``u*du`` and ``v*dv`` are formed on the host, and
``python/dpt/geometry_device.py:164-196`` for parallel and curved panels, whose
endpoints are formed per pixel from ``u, v, du, dv``).  A ``RayBundleGeometry``
is one view of explicit segments sharing one pose, as in the reference's
lower-level projector.
"""

from __future__ import annotations

import math
from collections.abc import Sequence
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .contracts import ContractError
from .geometry import (
    BatchedGeometry,
    CurvedDetectorGeometry,
    DetectorGeometry,
    ParallelGeometry,
    RayBundleGeometry,
)
from .volumes import GridSpec

GeometryInput = BatchedGeometry | DetectorGeometry | ParallelGeometry | CurvedDetectorGeometry


def batched(geometry: GeometryInput | Sequence[GeometryInput]) -> BatchedGeometry:
    """Normalise a panel, a sequence of panels or a ``BatchedGeometry``."""
    if isinstance(geometry, BatchedGeometry):
        return geometry
    if isinstance(geometry, (DetectorGeometry, ParallelGeometry, CurvedDetectorGeometry)):
        return BatchedGeometry((geometry,))
    if isinstance(geometry, Sequence) and not isinstance(geometry, (str, bytes)):
        return BatchedGeometry(tuple(geometry))
    raise ContractError("geometry must be a panel, a sequence of panels or a BatchedGeometry")


def panel_record(panel: DetectorGeometry | ParallelGeometry | CurvedDetectorGeometry) -> np.ndarray:
    """``DPT_VIEW_WORDS`` doubles describing one panel (layout in include/dpt_b200.h)."""
    record = np.zeros(N.VIEW_WORDS, dtype=np.float64)
    if isinstance(panel, ParallelGeometry):
        record[0:3] = panel.direction
        record[3:6] = panel.origin_mm
        record[6:9] = panel.u
        record[9:12] = panel.v
        record[12:14] = panel.spacing_mm
        record[14] = panel.length_mm
        record[N.VIEW_MODE_WORD] = N.PANEL_PARALLEL
    elif isinstance(panel, CurvedDetectorGeometry):
        record[0:3] = panel.source_mm
        record[3:6] = panel.origin_mm
        record[6:9] = panel.u
        record[9:12] = panel.v
        record[12:14] = panel.spacing_mm
        record[14] = panel.radius_mm
        record[15:18] = panel.radial_mm
        record[N.VIEW_MODE_WORD] = N.PANEL_CURVED
    elif isinstance(panel, DetectorGeometry):
        record[0:3] = panel.source_mm
        record[3:6] = panel.origin_mm
        record[6:9] = [x * panel.spacing_mm[0] for x in panel.u]
        record[9:12] = [x * panel.spacing_mm[1] for x in panel.v]
        record[N.VIEW_MODE_WORD] = N.PANEL_CONE
    else:
        raise ContractError("unsupported panel geometry")
    return record


@dataclass(frozen=True)
class RayPlan:
    """Flat description of one grid and acquisition."""

    grid: GridSpec
    views: int
    rows: int
    cols: int
    ray_kind: int
    object_to_grid: tuple[float, ...]
    grid_origin: tuple[float, ...]
    view_table: np.ndarray | None = field(default=None, repr=False)
    sources: np.ndarray | None = field(default=None, repr=False)
    endpoints: np.ndarray | None = field(default=None, repr=False)

    @property
    def rays_per_view(self) -> int:
        return self.rows * self.cols

    @property
    def rays(self) -> int:
        return self.views * self.rows * self.cols

    @property
    def image_shape(self) -> tuple[int, ...]:
        if self.ray_kind == N.RAYS_BUNDLE:
            return (self.cols,)
        return (self.views, self.rows, self.cols)

    def problem(
        self,
        samples: int,
        arith: int,
        *,
        field_dtype: int = N.F32,
        image_dtype: int = N.F32,
        layout: int = N.LAYOUT_REPLICATED,
        block_cols: int = 0,
        field_domain: int = N.DOMAIN_PHYSICAL,
    ) -> N.Problem:
        nz, ny, nx = self.grid.shape
        p = N.Problem()
        p.nx, p.ny, p.nz = nx, ny, nz
        p.views, p.rows, p.cols = self.views, self.rows, self.cols
        p.samples = samples
        p.ray_kind = self.ray_kind
        p.arith = arith
        p.field_dtype = field_dtype
        p.image_dtype = image_dtype
        p.layout = layout
        p.block_cols = block_cols
        p.field_domain = field_domain
        for k in range(9):
            p.object_to_grid[k] = self.object_to_grid[k]
        for k in range(3):
            p.grid_origin[k] = self.grid_origin[k]
        return p


def _grid_map(grid: GridSpec) -> tuple[tuple[float, ...], tuple[float, ...]]:
    matrix = grid.object_to_grid_matrix()
    if not all(math.isfinite(x) for x in matrix):
        raise ContractError("grid spacing overflows the FP64 coordinate map")
    return matrix, tuple(grid.origin_mm)


def plan_rays(grid: GridSpec, geometry: GeometryInput | RayBundleGeometry | Sequence) -> RayPlan:
    """Build the flat plan for ``grid`` and a panel batch or an explicit ray bundle."""
    if not isinstance(grid, GridSpec):
        raise ContractError("grid must be a GridSpec")
    matrix, origin = _grid_map(grid)
    if isinstance(geometry, RayBundleGeometry):
        sources = np.ascontiguousarray(np.asarray(geometry.sources_mm, dtype=np.float64))
        endpoints = np.ascontiguousarray(np.asarray(geometry.endpoints_mm, dtype=np.float64))
        return RayPlan(
            grid, 1, 1, geometry.pixels, N.RAYS_BUNDLE, matrix, origin,
            sources=sources, endpoints=endpoints,
        )
    batch = batched(geometry)
    for panel in batch.views:
        if isinstance(panel, DetectorGeometry):
            rows, cols = panel.shape
            for row in (0, rows - 1):
                for column in (0, cols - 1):
                    end = panel.pixel_centre(row, column)
                    if not all(math.isfinite(x) for x in end) or not math.isfinite(
                        math.dist(end, panel.source_mm)
                    ):
                        raise ContractError("detector extent exceeds the FP64 finite-ray range")
    table = np.ascontiguousarray(np.stack([panel_record(panel) for panel in batch.views]))
    rows, cols = batch.shape_rows_columns
    return RayPlan(grid, len(batch.views), rows, cols, N.RAYS_PANELS, matrix, origin, view_table=table)
