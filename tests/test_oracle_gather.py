"""The oracle's deterministic adjoint gather pinned to the reference's independent FP64
midpoint matrices (``golden/make_gather_golden.py``: the scenes of the reference's gather
tests, matrices from its scalar oracle ``validation/projection.py``), with the reference's own
bar: A^T s within 2e-12, the adjoint identity <A v, s> = <v, A^T s> within 2e-12, repeatable
bit for bit, accumulation and FP32 output as a per-view loop forms them.  Oracle-only: no GPU.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from dpt_b200.geometry import BatchedGeometry
from dpt_b200.plan import plan_rays
from oracle import oracle as O
from scenes import gather_matrix, gather_scene


@pytest.mark.parametrize("name", ["gather_nonsquare", "gather_bundle", "gather_clamped", "culled_tilted"])
def test_gather_matches_reference_matrix_and_adjoint_pairs(name):
    grid, geometry, pose, samples = gather_scene(name)
    plan = plan_rays(grid, geometry)
    matrix = gather_matrix(name)
    rng = np.random.default_rng(584291)
    for _ in range(5):
        values = rng.uniform(-1, 1, grid.voxels).astype(np.float32)
        seeds = rng.uniform(-1, 1, plan.rays)
        gradient, status = O.gather(plan, pose, seeds, samples=samples)
        assert status == 0
        expected = matrix.T @ seeds
        np.testing.assert_allclose(gradient, expected, rtol=2e-12, atol=2e-12)
        image, _ = O.forward(plan, values, pose, samples=samples, arith=O.ARITH_F64, image_dtype=O.F64)
        left = math.fsum(image * seeds)
        right = math.fsum(values.astype(np.float64) * gradient)
        assert abs(left - right) < 2e-12 * max(1.0, abs(left), abs(right))
        again, _ = O.gather(plan, pose, seeds, samples=samples)
        assert again.tobytes() == gradient.tobytes()


def test_accumulation_fp32_output_and_views_in_order():
    grid, geometry, pose, samples = gather_scene("culled_tilted")
    views = BatchedGeometry((geometry, geometry, geometry))
    plan = plan_rays(grid, views)
    single = plan_rays(grid, geometry)
    rng = np.random.default_rng(3)
    seeds = rng.normal(size=(3, single.rays))
    seeds[:, ::4] = 0.0
    for dtype, cast in ((O.F64, np.float64), (O.F32, np.float32)):
        running = None
        for view in range(3):
            running, _ = O.gather(single, pose, seeds[view], samples=samples, out_dtype=dtype, out=running,
                                  accumulate=running is not None)
        together, status = O.gather(plan, pose, seeds.reshape(-1), samples=samples, out_dtype=dtype)
        assert status == 0 and together.dtype == cast
        assert together.tobytes() == running.tobytes()
        doubled, _ = O.gather(plan, pose, seeds.reshape(-1), samples=samples, out_dtype=dtype, out=together,
                              accumulate=True)
        scale = float(np.abs(together).max())
        np.testing.assert_allclose(doubled, 2 * together, rtol=0, atol=(4e-7 if dtype == O.F32 else 1e-15) * scale)


def test_overflowing_zero_weight_corner_keeps_the_canonical_failure():
    """A clamped corner of zero weight times an overflowing cotangent is NaN, as the reference
    sums it (tests/python/warp_cpu/test_projection_culled_adjoint.py:433-451)."""
    from dpt_b200.geometry import RayBundleGeometry
    from dpt_b200.volumes import GridSpec

    grid = GridSpec((1, 1, 2), (10.0, 1.0, 1.0))
    plan = plan_rays(grid, RayBundleGeometry(((-100.0, 0.0, 0.0),), ((0.0, 0.0, 0.0),)))
    pose = np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0])
    gradient, status = O.gather(plan, pose, np.array([1e308]), samples=1)
    assert status & 2
    assert np.isnan(gradient).all()


@pytest.mark.parametrize("name", ["gather_nonsquare", "gather_bundle", "gather_clamped"])
def test_cell_gauss_gather_matches_reference_exact_matrix(name):
    grid, geometry, pose, _ = gather_scene(name)
    plan = plan_rays(grid, geometry)
    matrix = np.load(__import__("scenes").GOLDEN / "gather.npz")[f"{name}_cells_matrix"]
    rng = np.random.default_rng(91)
    for _ in range(5):
        values = rng.uniform(-1, 1, grid.voxels).astype(np.float32)
        seeds = rng.uniform(-1, 1, plan.rays)
        gradient, status = O.gather(plan, pose, seeds, samples=1, cells=True)
        assert status == 0
        np.testing.assert_allclose(gradient, matrix.T @ seeds, rtol=2e-12, atol=2e-12)
        image, _ = O.forward(plan, values, pose, samples=1, arith=O.ARITH_CELLS, image_dtype=O.F64)
        left, right = math.fsum(image * seeds), math.fsum(values.astype(np.float64) * gradient)
        assert abs(left - right) < 2e-12 * max(1.0, abs(left), abs(right))
