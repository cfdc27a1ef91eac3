"""Generate ``gather.npz`` / ``gather.json``: the scenes of the reference's deterministic-gather
tests and their independent FP64 midpoint matrices.  Run with the reference checkout given
by ``--reference PATH`` or ``DPT_REFERENCE`` (its host code imports without Warp):

    python tests/golden/make_gather_golden.py --reference PATH

Sources used (paths inside the reference project):
  * tests/python/warp_cpu/test_projection_adjoint_gather.py:26-74 ``_metadata`` (scenes
    "nonsquare", "bundle", "clamped"); the 31-sample midpoint and the cell-Gauss matrices are
    formed as its ``_matrix`` (:75-96) forms them, from python/dpt/validation/projection.py
    ``integrate_sampled_field`` / ``integrate_ray_bundle``
  * tests/python/warp_cpu/test_projection_culled_adjoint.py:91-138 ``_scene`` (kinds "tilted",
    "inside", "negative_depth", "underflow_plane", "tolerated_rotation", "bundle", and the
    singleton-axis shapes) and the 37-sample matrix of its "tilted" scene (:325-335)
The test helpers are extracted from their files with ``ast`` and executed with the reference's
modules, because the test modules import Warp at top level.
"""

from __future__ import annotations

import ast
import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from reference_checkout import reference_root  # noqa: E402

REFERENCE = reference_root()

from dpt import geometry as rg  # noqa: E402
from dpt.validation import projection as rv  # noqa: E402
from dpt.volumes import GridSpec  # noqa: E402


def extract(path: Path, names: list[str], namespace: dict) -> dict:
    tree = ast.parse(path.read_text())
    keep = [node for node in tree.body if isinstance(node, ast.FunctionDef) and node.name in names]
    missing = set(names) - {node.name for node in keep}
    if missing:
        raise RuntimeError(f"{path}: missing {missing}")
    exec(compile(ast.Module(body=keep, type_ignores=[]), str(path), "exec"), namespace)
    return namespace


def grid_record(grid: GridSpec) -> dict:
    return {"shape": list(grid.shape), "spacing_mm": list(grid.spacing_mm), "origin_mm": list(grid.origin_mm),
            "orientation": list(grid.orientation)}


def geometry_record(geometry) -> dict:
    if isinstance(geometry, rg.RayBundleGeometry):
        return {"kind": "bundle", "sources_mm": [list(s) for s in geometry.sources_mm],
                "endpoints_mm": [list(e) for e in geometry.endpoints_mm]}
    return {"kind": "cone", "source_mm": list(geometry.source_mm), "origin_mm": list(geometry.origin_mm),
            "u": list(geometry.u), "v": list(geometry.v), "spacing_mm": list(geometry.spacing_mm),
            "shape": list(geometry.shape)}


def scalar_matrix(grid, geometry, pose, samples: int | None) -> np.ndarray:
    """Pixels x voxels FP64 matrix from the reference's scalar oracle: midpoint with `samples`,
    or the exact piecewise (cell-Gauss) integral for None."""
    matrix = np.empty((geometry.pixels, grid.voxels))
    for voxel in range(grid.voxels):
        basis = [float(index == voxel) for index in range(grid.voxels)]
        for pixel in range(geometry.pixels):
            if isinstance(geometry, rg.RayBundleGeometry):
                matrix[pixel, voxel] = rv.integrate_ray_bundle(basis, grid, geometry, pose, pixel,
                                                               midpoint_samples=samples)
            else:
                row, column = divmod(pixel, geometry.shape[1])
                matrix[pixel, voxel] = rv.integrate_sampled_field(basis, grid, geometry, pose, row, column,
                                                                  midpoint_samples=samples)
    return matrix


def main() -> None:
    common = {"math": math, "GridSpec": GridSpec, "DetectorGeometry": rg.DetectorGeometry,
              "RayBundleGeometry": rg.RayBundleGeometry, "RigidTransform": rg.RigidTransform,
              "compose_pose": rg.compose_pose, "integrate_ray_bundle": rv.integrate_ray_bundle,
              "integrate_sampled_field": rv.integrate_sampled_field}
    gather_tests = extract(REFERENCE / "tests/python/warp_cpu/test_projection_adjoint_gather.py",
                           ["_metadata"], dict(common))
    culled_tests = extract(REFERENCE / "tests/python/warp_cpu/test_projection_culled_adjoint.py",
                           ["_scene"], dict(common))
    cases, arrays = {}, {}
    for case in ("nonsquare", "bundle", "clamped"):
        grid, geometry, pose = gather_tests["_metadata"](case)
        name = f"gather_{case}"
        cases[name] = {"grid": grid_record(grid), "geometry": geometry_record(geometry),
                       "pose": list(pose.packed()), "samples": 31}
        arrays[f"{name}_matrix"] = scalar_matrix(grid, geometry, pose, 31)
        arrays[f"{name}_cells_matrix"] = scalar_matrix(grid, geometry, pose, None)
    kinds = ["tilted", "inside", "negative_depth", "underflow_plane", "tolerated_rotation", "bundle"]
    for kind in kinds:
        grid, geometry, pose = culled_tests["_scene"](kind)
        cases[f"culled_{kind}"] = {"grid": grid_record(grid), "geometry": geometry_record(geometry),
                                   "pose": list(pose.packed()), "samples": 37}
    grid, geometry, pose = culled_tests["_scene"]("tilted")
    arrays["culled_tilted_matrix"] = scalar_matrix(grid, geometry, pose, 37)
    for shape in [(1, 2, 3), (1, 3, 2), (2, 1, 3), (3, 1, 2), (2, 3, 1), (3, 2, 1)]:
        grid, geometry, pose = culled_tests["_scene"]("tilted", shape)
        cases["singleton_" + "x".join(map(str, shape))] = {
            "grid": grid_record(grid), "geometry": geometry_record(geometry), "pose": list(pose.packed()),
            "samples": 37}
    grid, geometry, pose = culled_tests["_scene"]("large_tilted")
    cases["culled_large_tilted"] = {"grid": grid_record(grid), "geometry": geometry_record(geometry),
                                    "pose": list(pose.packed()), "samples": 37}
    np.savez_compressed(HERE / "gather.npz", **arrays)
    (HERE / "gather.json").write_text(json.dumps(cases, indent=1))
    print(sorted(cases), {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
