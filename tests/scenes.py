"""Seeded scenes shared by the tests: golden fixtures and small cone-beam scans."""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

from dpt_b200.geometry import (
    BatchedGeometry,
    ConeBeamIntrinsics,
    CurvedDetectorGeometry,
    DetectorGeometry,
    ParallelGeometry,
    RayBundleGeometry,
    RigidTransform,
    compose_pose,
)
from dpt_b200.phantoms import centred_grid, ellipsoid_phantom
from dpt_b200.volumes import GridSpec

GOLDEN = Path(__file__).resolve().parent / "golden"


def grid_from(record: dict) -> GridSpec:
    return GridSpec(tuple(record["shape"]), tuple(record["spacing_mm"]), tuple(record["origin_mm"]),
                    tuple(record["orientation"]))


def panel_from(record: dict) -> DetectorGeometry:
    return DetectorGeometry(tuple(record["source_mm"]), tuple(record["origin_mm"]), tuple(record["u"]),
                            tuple(record["v"]), tuple(record["spacing_mm"]), tuple(record["shape"]))


def fp32_fixture():
    """5x6x7 oriented grid, five explicit rays, one pose (reference FP32 matrix scene)."""
    data = np.load(GOLDEN / "fp32_matrix.npz")
    grid = grid_from(json.loads((GOLDEN / "fp32_matrix.json").read_text())["grid"])
    rays = RayBundleGeometry(tuple(map(tuple, data["sources"])), tuple(map(tuple, data["endpoints"])))
    return grid, rays, data


def projector_fixture():
    meta = json.loads((GOLDEN / "projector.json").read_text())
    data = np.load(GOLDEN / "projector.npz")
    grid = grid_from(meta["grid"])
    geometry = BatchedGeometry(tuple(panel_from(p) for p in meta["panels"]))
    return grid, geometry, data, meta["samples"]


def native_fixture():
    meta = json.loads((GOLDEN / "native_storage.json").read_text())
    data = np.load(GOLDEN / "native_storage.npz")
    grid = grid_from(meta["grid"])
    rays = RayBundleGeometry(tuple(map(tuple, data["sources"])), tuple(map(tuple, data["endpoints"])))
    return grid, rays, data, meta["samples"]


def rotated_grid(shape, spacing, angle=0.3):
    c, s = math.cos(angle), math.sin(angle)
    return centred_grid(shape, spacing, (c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0))


def cone_scene(shape=(14, 16, 18), spacing=(1.3, 1.1, 1.2), views=4, detector=(20, 24),
               pitch=(2.0, 2.0), seed=5, sod=60.0, sdd=110.0, angle=0.3):
    """Small oriented grid, additive ellipsoids and a circular cone scan."""
    grid = rotated_grid(shape, spacing, angle)
    values, _ = ellipsoid_phantom(grid, seed=seed, count=4)
    intrinsics = ConeBeamIntrinsics(sod, sdd, detector, pitch, (0.7, -0.45), (0.3, -0.2, 0.1))
    angles = tuple(2 * math.pi * k / views + 0.11 for k in range(views))
    return grid, intrinsics.batch(angles), values


def config1_scene(seed=0):
    """64^3 1 mm ellipsoid phantom, 8 cone views over 360 deg, SOD 500, SDD 1000, 64x64 at 1.5 mm."""
    grid = centred_grid((64, 64, 64), (1.0, 1.0, 1.0))
    values, _ = ellipsoid_phantom(grid, seed=seed)
    intrinsics = ConeBeamIntrinsics(500.0, 1000.0, (64, 64), (1.5, 1.5))
    geometry = intrinsics.batch(tuple(2 * math.pi * k / 8 for k in range(8)))
    return grid, geometry, values


def mixed_panels(grid: GridSpec, shape=(9, 11)):
    """One cone, one parallel and one curved panel around the grid."""
    cone = ConeBeamIntrinsics(50.0, 90.0, shape, (2.2, 2.0)).view(0.4)
    parallel = ParallelGeometry((-12.0, 30.0, -9.0), (0.0, 1.0, 0.0), 70.0, (1.0, 0.0, 0.0), (0.0, 0.0, 1.0),
                                (2.1, 1.9), shape)
    # cylinder through the source along z; first pixel on the radius 80 circle
    source = (0.0, -45.0, 0.0)
    start = -0.5 * (shape[1] - 1) * 2.0 / 80.0
    origin = (80.0 * math.sin(start), -45.0 + 80.0 * math.cos(start), -0.5 * (shape[0] - 1) * 2.0)
    u = (math.cos(start), -math.sin(start), 0.0)
    curved = CurvedDetectorGeometry(source, origin, u, (0.0, 0.0, 1.0), (2.0, 2.0), shape)
    return BatchedGeometry((cone, parallel, curved))


def poses_for(views: int, seed: int = 1, scale: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(views):
        xi = tuple(float(x) for x in rng.normal(size=6) * scale * np.array([10, 10, 10, 1, 1, 1]))
        out.append(compose_pose(RigidTransform(), xi).packed())
    return np.asarray(out, dtype=np.float64)


def identity_poses(views: int) -> np.ndarray:
    return np.tile(np.asarray(RigidTransform().packed()), (views, 1))


def gather_scene(name: str):
    """(grid, geometry, packed pose, samples) of a deterministic-gather golden scene."""
    record = json.loads((GOLDEN / "gather.json").read_text())[name]
    geometry = record["geometry"]
    if geometry["kind"] == "bundle":
        panel = RayBundleGeometry(tuple(tuple(s) for s in geometry["sources_mm"]),
                                  tuple(tuple(e) for e in geometry["endpoints_mm"]))
    else:
        panel = panel_from(geometry)
    return grid_from(record["grid"]), panel, np.asarray(record["pose"], dtype=np.float64), record["samples"]


def gather_matrix(name: str) -> np.ndarray:
    return np.load(GOLDEN / "gather.npz")[f"{name}_matrix"]
