"""Generate the golden fixtures in this directory from the reference projector's own
pure-Python oracles.  Run with the reference checkout given by ``--reference PATH`` or
``DPT_REFERENCE`` (its host code imports without Warp):

    python tests/golden/make_golden.py --reference PATH

Sources used (paths inside the reference project):
  * python/dpt/validation/projection.py   - FP64 midpoint / exact piecewise-Gauss integrals
  * tests/python/warp_cpu/test_projection_fp32.py:24-119
        ``_scene`` and ``_matrix``: the independent numpy FP32 weight matrix
  * tests/python/warp_cpu/test_projector_workflow.py:28-60
        ``_problem`` and ``_matrix``: Projector scene and FP64 midpoint matrix
  * tests/python/warp_cpu/test_projection_native_storage.py:33-84
        ``_metadata`` and ``_float32_oracle``: FP32-marching oracle on decoded half storage
  * tests/python/test_projection_reference.py: closed-form integrals
  * python/dpt/phantoms.py: analytic ellipsoid chords
  * python/dpt/geometry.py: compose_pose / right_jacobian_se3 / chart_gradient, cone views
  * benchmarks/fullscan_guards.py:15-55: numpy FP64 reference ray
The test helpers are extracted from their files with ``ast`` and executed with the
reference's modules, because the test modules themselves import Warp at top level.
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
from dpt import phantoms as rp  # noqa: E402
from dpt.validation import projection as rv  # noqa: E402
from dpt.volumes import GridSpec  # noqa: E402


def extract(path: Path, names: list[str], namespace: dict) -> dict:
    """Execute the named top-level functions of a reference test file in `namespace`."""
    tree = ast.parse(path.read_text())
    keep = [node for node in tree.body if isinstance(node, ast.FunctionDef) and node.name in names]
    missing = set(names) - {node.name for node in keep}
    if missing:
        raise RuntimeError(f"{path}: missing {missing}")
    module = ast.Module(body=keep, type_ignores=[])
    exec(compile(module, str(path), "exec"), namespace)
    return namespace


def grid_record(grid: GridSpec) -> dict:
    return {
        "shape": list(grid.shape),
        "spacing_mm": list(grid.spacing_mm),
        "origin_mm": list(grid.origin_mm),
        "orientation": list(grid.orientation),
    }


def fp32_matrix_fixture() -> None:
    """Reference FP32 numpy weight matrix on the 5x6x7 oriented scene."""
    ns = extract(
        REFERENCE / "tests/python/warp_cpu/test_projection_fp32.py",
        ["_scene", "_fma32", "_matrix"],
        {
            "np": np,
            "math": math,
            "GridSpec": GridSpec,
            "RayBundleGeometry": rg.RayBundleGeometry,
            "RigidTransform": rg.RigidTransform,
            "compose_pose": rg.compose_pose,
            "_clip_segment": rv._clip_segment,
        },
    )
    grid, rays, pose, values = ns["_scene"]()
    out = {
        "values": values,
        "pose": np.asarray(pose.packed()),
        "sources": np.asarray(rays.sources_mm),
        "endpoints": np.asarray(rays.endpoints_mm),
        "seeds": np.asarray([0.7, -0.3, 0.2, 0.6, 1.0], dtype=np.float32),
    }
    for samples in (17, 97, 1024):
        matrix = ns["_matrix"](grid, rays, pose, samples)
        out[f"matrix_{samples}"] = matrix
    np.savez_compressed(HERE / "fp32_matrix.npz", **out)
    (HERE / "fp32_matrix.json").write_text(json.dumps({"grid": grid_record(grid)}, indent=1))


def projector_fixture() -> None:
    """Projector workflow scene and its FP64 47-sample midpoint matrix."""
    import torch

    ns = extract(
        REFERENCE / "tests/python/warp_cpu/test_projector_workflow.py",
        ["_problem", "_matrix"],
        {
            "torch": torch,
            "GridSpec": GridSpec,
            "DetectorGeometry": rg.DetectorGeometry,
            "BatchedGeometry": rg.BatchedGeometry,
            "RigidTransform": rg.RigidTransform,
            "replace": __import__("dataclasses").replace,
            "integrate_sampled_field": rv.integrate_sampled_field,
        },
    )
    grid, geometry, field = ns["_problem"]("cpu")
    matrix = ns["_matrix"](grid, geometry, "cpu").numpy()
    panels = [
        {
            "source_mm": list(p.source_mm),
            "origin_mm": list(p.origin_mm),
            "u": list(p.u),
            "v": list(p.v),
            "spacing_mm": list(p.spacing_mm),
            "shape": list(p.shape),
        }
        for p in geometry.views
    ]
    np.savez_compressed(HERE / "projector.npz", field=field.numpy(), matrix_47=matrix)
    (HERE / "projector.json").write_text(
        json.dumps({"grid": grid_record(grid), "panels": panels, "samples": 47}, indent=1)
    )


def native_storage_fixture() -> None:
    """FP32-marching oracle on decoded FP16 / BF16 values (31 samples)."""
    import struct

    ns = extract(
        REFERENCE / "tests/python/warp_cpu/test_projection_native_storage.py",
        ["_f32", "_metadata", "_float32_oracle"],
        {
            "struct": struct,
            "math": math,
            "GridSpec": GridSpec,
            "RayBundleGeometry": rg.RayBundleGeometry,
            "RigidTransform": rg.RigidTransform,
            "_clip_segment": rv._clip_segment,
        },
    )
    grid, rays = ns["_metadata"]()
    original = np.asarray([0.07 + 0.003 * (voxel % 11) for voxel in range(grid.voxels)])
    out = {"sources": np.asarray(rays.sources_mm), "endpoints": np.asarray(rays.endpoints_mm)}
    import torch

    for name, dtype in (("float16", torch.float16), ("bfloat16", torch.bfloat16)):
        stored = torch.tensor(original, dtype=dtype)
        decoded = stored.float().numpy().astype(np.float64).tolist()
        image, matrix = ns["_float32_oracle"](decoded, grid, rays, 31)
        out[f"{name}_bits"] = stored.view(torch.int16).numpy().view(np.uint16)
        out[f"{name}_image"] = np.asarray(image)
        out[f"{name}_matrix"] = np.asarray(matrix)
    np.savez_compressed(HERE / "native_storage.npz", **out)
    (HERE / "native_storage.json").write_text(json.dumps({"grid": grid_record(grid), "samples": 31}, indent=1))


def closed_form_fixture() -> dict:
    """Closed-form integrals of tests/python/test_projection_reference.py and the
    clipped single-voxel case of tests/python/warp_cpu/test_projection_fp32.py:248-257."""

    def panel(source=-10.0, detector=10.0):
        return rg.DetectorGeometry(
            (source, 0.0, 0.0), (detector, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0), (1.0, 1.0), (1, 1)
        )

    identity = rg.RigidTransform()
    cases = []
    g1 = GridSpec((1, 1, 1), (2.0, 3.0, 4.0))
    cases.append({"grid": grid_record(g1), "values": [0.25], "source": -10.0, "detector": 10.0,
                  "gauss": rv.integrate_sampled_field([0.25], g1, panel(), identity, 0, 0)})
    g3 = GridSpec((1, 1, 3), (2.0, 1.0, 1.0))
    for source, detector, values in ((-10.0, 10.0, [1.0, 3.0, 2.0]), (0.0, 10.0, [0.5, 0.5, 0.5]),
                                     (-10.0, -3.0, [1.0, 1.0, 1.0])):
        p = panel(source, detector)
        cases.append({
            "grid": grid_record(g3), "values": values, "source": source, "detector": detector,
            "gauss": rv.integrate_sampled_field(values, g3, p, identity, 0, 0),
            "midpoint_7": rv.integrate_sampled_field(values, g3, p, identity, 0, 0, midpoint_samples=7),
            "midpoint_701": rv.integrate_sampled_field(values, g3, p, identity, 0, 0, midpoint_samples=701),
            "midpoint_1024": rv.integrate_sampled_field(values, g3, p, identity, 0, 0, midpoint_samples=1024),
        })
    quadratic_grid = GridSpec((1, 1, 3), (2.0, 1.0, 1.0), (-2.0, 0.0, 0.0))
    quadratic = rv.integrate_quadratic_field(
        quadratic_grid, panel(), identity, 0, 0, intercept=0.2, curvature=(0.1, 0.0, 0.0)
    )
    return {
        "cases": cases,
        "quadratic": {"grid": grid_record(quadratic_grid), "value": quadratic},
        "single_voxel": {"value": 0.025 * 0.7, "volume": 0.7, "tangent": [-0.025, 0, 0, 0, 0, 0]},
    }


def ellipsoid_fixture() -> dict:
    """Seeded ellipsoids, their sampled grid and analytic chords for a few rays."""
    rng = np.random.default_rng(20240611)
    models = []
    for _ in range(4):
        axes = tuple(float(x) for x in rng.uniform(5.0, 12.0, 3))
        angle = float(rng.uniform(0, math.pi))
        c, s = math.cos(angle), math.sin(angle)
        models.append(rp.Ellipsoid(axes, float(rng.uniform(0.01, 0.05)),
                                   tuple(float(x) for x in rng.uniform(-6, 6, 3)),
                                   (c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0)))
    grid = GridSpec((48, 48, 48), (0.75, 0.75, 0.75), (-17.625, -17.625, -17.625))
    values = rp.sample_ellipsoids(grid, models)
    panels = rp.circular_cone_beam((0.0, 1.1, 2.3), source_radius_mm=120.0, detector_radius_mm=80.0,
                                   shape_rows_columns=(9, 11), spacing_column_row_mm=(3.0, 3.0))
    chords = []
    for panel in panels:
        for row in range(panel.shape[0]):
            for column in range(panel.shape[1]):
                end = panel.pixel_centre(row, column)
                chords.append(sum(m.optical_depth(panel.source_mm, end) for m in models))
    np.savez_compressed(HERE / "ellipsoids.npz", values=values, chords=np.asarray(chords))
    return {
        "grid": grid_record(grid),
        "models": [{"axes_mm": list(m.axes_mm), "mu": m.attenuation_mm_inverse,
                    "centre_mm": list(m.centre_mm), "orientation": list(m.orientation)} for m in models],
        "panels": [{"source_mm": list(p.source_mm), "origin_mm": list(p.origin_mm), "u": list(p.u),
                    "v": list(p.v), "spacing_mm": list(p.spacing_mm), "shape": list(p.shape)} for p in panels],
    }


def chart_fixture() -> dict:
    rng = np.random.default_rng(7)
    out = []
    anchor = rg.RigidTransform((0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0), (3.0, -2.0, 1.0))
    for scale in (1e-4, 1e-2, 0.3, 1.5):
        xi = tuple(float(x) for x in rng.normal(size=6) * scale)
        g = tuple(float(x) for x in rng.normal(size=6))
        out.append({
            "increment": list(xi),
            "composed": list(rg.compose_pose(anchor, xi).packed()),
            "jacobian": [list(row) for row in rg.right_jacobian_se3(xi)],
            "right_gradient": list(g),
            "chart_gradient": list(rg.chart_gradient(xi, g)),
        })
    return {"anchor": list(anchor.packed()), "cases": out}


def cone_fixture() -> dict:
    intrinsics = rg.ConeBeamIntrinsics(500.0, 1000.0, (64, 64), (1.5, 1.5), (0.7, -0.4), (1.0, 2.0, 3.0))
    views = []
    for angle in (0.0, 0.7, 2.0, 4.5):
        panel = intrinsics.view(angle)
        views.append({"angle": angle, "source_mm": list(panel.source_mm), "origin_mm": list(panel.origin_mm),
                      "u": list(panel.u), "v": list(panel.v), "centre_3_5": list(panel.pixel_centre(3, 5)),
                      "project_point": list(panel.project_point((10.0, -4.0, 7.0)))})
    from dpt.imaging import standard_views

    grid = GridSpec((20, 30, 40), (0.9, 0.8, 2.0), (-5.0, 3.0, 1.0))
    std = standard_views(grid, shape=(32, 48))
    return {
        "views": views,
        "standard_views": [{"source_mm": list(p.source_mm), "origin_mm": list(p.origin_mm), "u": list(p.u),
                            "v": list(p.v), "spacing_mm": list(p.spacing_mm)} for p in std.views],
        "standard_grid": grid_record(grid),
    }


def guard_fixture() -> dict:
    """numpy FP64 reference rays of benchmarks/fullscan_guards.py on a small volume."""
    from benchmarks.fullscan_guards import reference_ray

    rng = np.random.default_rng(3)
    grid = GridSpec((12, 14, 16), (1.1, 0.9, 1.3), (-8.0, -6.0, -7.0))
    values = rng.uniform(0.0, 0.05, grid.shape).astype(np.float32)
    intrinsics = rg.ConeBeamIntrinsics(200.0, 320.0, (10, 12), (2.0, 2.0))
    pose = rg.compose_pose(rg.RigidTransform(), (0.3, -0.2, 0.4, 0.05, -0.03, 0.02))
    rays = []
    for angle in (0.0, 1.3):
        panel = intrinsics.view(angle)
        for row, column in ((0, 0), (5, 6), (9, 11), (3, 8)):
            rays.append(reference_ray(values.astype(np.float64), grid, panel, pose, row, column, 256))
    np.savez_compressed(HERE / "guard.npz", values=values, rays=np.asarray(rays))
    return {"grid": grid_record(grid), "pose": list(pose.packed()), "angles": [0.0, 1.3],
            "pixels": [[0, 0], [5, 6], [9, 11], [3, 8]], "samples": 256}


def main() -> None:
    fp32_matrix_fixture()
    projector_fixture()
    native_storage_fixture()
    facts = {
        "closed_form": closed_form_fixture(),
        "ellipsoids": ellipsoid_fixture(),
        "chart": chart_fixture(),
        "cone": cone_fixture(),
        "guard": guard_fixture(),
    }
    (HERE / "facts.json").write_text(json.dumps(facts, indent=1))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
