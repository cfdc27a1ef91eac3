"""The CPU oracle pinned against the reference projector's own oracles and known answers.

Fixtures in tests/golden were produced by tests/golden/make_golden.py from the
reference's pure-Python oracles (FP64 midpoint / Gauss integrals, the numpy FP32
weight matrix of its FP32 tests, its half-storage FP32 oracle, analytic chords).
Tolerances are the reference tests' own where they have one.
"""

from __future__ import annotations

import json
import math

import numpy as np
import pytest

from dpt_b200.geometry import (
    BatchedGeometry,
    DetectorGeometry,
    RayBundleGeometry,
    RigidTransform,
    compose_pose,
)
from dpt_b200.plan import plan_rays
from dpt_b200.volumes import GridSpec
from oracle import oracle as O
from scenes import GOLDEN, fp32_fixture, grid_from, native_fixture, panel_from, projector_fixture

FACTS = json.loads((GOLDEN / "facts.json").read_text())
IDENTITY = np.asarray(RigidTransform().packed())


@pytest.mark.parametrize("samples", [17, 97, 1024])
def test_fp32_forward_and_volume_vjp_match_reference_weight_matrix(samples):
    """Reference tests/python/warp_cpu/test_projection_fp32.py:122-134 (rtol 2e-5, atol 3e-7)."""
    grid, rays, data = fp32_fixture()
    plan = plan_rays(grid, rays)
    matrix = data[f"matrix_{samples}"]
    values = data["values"].astype(np.float64)
    image, status = O.forward(plan, data["values"], data["pose"], samples=samples)
    assert not status.any()
    np.testing.assert_allclose(image, matrix @ values, rtol=2e-5, atol=3e-7)
    volume, _, _ = O.vjp(plan, data["values"], data["pose"], data["seeds"], samples=samples, flags=O.VJP_VOLUME)
    np.testing.assert_allclose(volume, matrix.T @ data["seeds"].astype(np.float64), rtol=2e-5, atol=3e-7)
    left, right = float(image.astype(np.float64) @ data["seeds"]), float(values @ volume)
    assert abs(left - right) / max(abs(left), abs(right)) < 1e-5


def test_fp32_pose_matches_strict_pose_and_finite_differences():
    """Reference test_projection_fp32.py:137-164: FP32 vs strict (2e-3 / 1e-5) and FD (< 1e-2)."""
    grid, rays, data = fp32_fixture()
    plan = plan_rays(grid, rays)
    seeds = np.asarray([0.7, -0.3, 0.2, 0.6, 0.0], dtype=np.float32)
    _, tangent, _ = O.vjp(plan, data["values"], data["pose"], seeds, samples=97, flags=O.VJP_POSE6)
    _, strict, _ = O.vjp(plan, data["values"], data["pose"], seeds.astype(np.float64), samples=97,
                         flags=O.VJP_POSE6, arith=O.ARITH_F64, image_dtype=O.F64)
    np.testing.assert_allclose(tangent[0], strict[0], rtol=2e-3, atol=1e-5)
    pose = RigidTransform(tuple(data["pose"][:9]), tuple(data["pose"][9:]))
    for direction in (np.asarray([0.4, -0.2, 0.3, 0.01, -0.02, 0.015]),
                      np.asarray([0.02, 0.03, -0.04, 0.15, -0.11, 0.07])):
        expected = float(tangent[0] @ direction)
        errors = []
        for eps in (3e-2, 1e-2, 3e-3, 1e-3):
            losses = []
            for sign in (-1, 1):
                shifted = compose_pose(pose, tuple(sign * eps * direction))
                image, _ = O.forward(plan, data["values"], np.asarray(shifted.packed()), samples=97)
                losses.append(float(image.astype(np.float64) @ seeds))
            errors.append(abs((losses[1] - losses[0]) / (2 * eps) - expected) / max(abs(expected), 1e-12))
        assert min(errors) < 1e-2, errors


def test_clipped_single_voxel_known_answer():
    """Reference test_projection_fp32.py:248-257: L = 0.025 * 0.7, dL/dmu = 0.7, pose (-0.025, 0...)."""
    grid = GridSpec((1, 1, 1), (1.0, 1.0, 1.0))
    plan = plan_rays(grid, RayBundleGeometry(((-2.0, 0.0, 0.0),), ((0.2, 0.0, 0.0),)))
    facts = FACTS["closed_form"]["single_voxel"]
    image, _ = O.forward(plan, np.asarray([0.025], np.float32), IDENTITY, samples=1024)
    np.testing.assert_allclose(image, [facts["value"]], rtol=2e-5)
    volume, tangent, _ = O.vjp(plan, np.asarray([0.025], np.float32), IDENTITY, np.ones(1, np.float32),
                               samples=1024, flags=O.VJP_VOLUME | O.VJP_POSE6)
    np.testing.assert_allclose(volume, [facts["volume"]], rtol=2e-5)
    np.testing.assert_allclose(tangent[0], facts["tangent"], rtol=2e-5, atol=1e-8)


def _line_panel(source: float, detector: float) -> DetectorGeometry:
    return DetectorGeometry((source, 0.0, 0.0), (detector, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0),
                            (1.0, 1.0), (1, 1))


@pytest.mark.parametrize("index", range(4))
def test_closed_form_integrals(index):
    """Reference tests/python/test_projection_reference.py: half-cell margins, truncation,
    detector before support, midpoint -> exact convergence."""
    case = FACTS["closed_form"]["cases"][index]
    grid = grid_from(case["grid"])
    plan = plan_rays(grid, _line_panel(case["source"], case["detector"]))
    values = np.asarray(case["values"], dtype=np.float32)
    for samples, key in ((7, "midpoint_7"), (701, "midpoint_701"), (1024, "midpoint_1024")):
        if key not in case:
            continue
        image64, _ = O.forward(plan, values, IDENTITY, samples=samples, arith=O.ARITH_F64, image_dtype=O.F64)
        assert image64[0] == pytest.approx(case[key], rel=1e-12, abs=1e-14)
        image32, _ = O.forward(plan, values, IDENTITY, samples=samples)
        assert image32[0] == pytest.approx(case[key], rel=2e-5, abs=1e-6)
    # fine midpoint rules converge to the exact piecewise-Gauss integral
    image, _ = O.forward(plan, values, IDENTITY, samples=4096, arith=O.ARITH_F64, image_dtype=O.F64)
    assert image[0] == pytest.approx(case["gauss"], rel=1e-5, abs=1e-9)
    # and cell-Gauss integration is that integral (reference validation/projection.py)
    cells, status = O.forward(plan, values, IDENTITY, samples=1, arith=O.ARITH_CELLS, image_dtype=O.F64)
    assert not status.any()
    assert cells[0] == pytest.approx(case["gauss"], rel=1e-12, abs=1e-14)


def test_projector_scene_matches_reference_fp64_matrix():
    """Reference test_projector_workflow.py:62-84: FP32 5e-6, FP64 2e-11 against the FP64 matrix."""
    grid, geometry, data, samples = projector_fixture()
    plan = plan_rays(grid, geometry)
    field = data["field"]
    matrix = data["matrix_47"]
    expected = matrix @ field.reshape(-1).astype(np.float64)
    poses = np.tile(IDENTITY, (len(geometry.views), 1))
    image64, _ = O.forward(plan, field, poses, samples=samples, arith=O.ARITH_F64, image_dtype=O.F64)
    np.testing.assert_allclose(image64, expected, rtol=2e-11, atol=2e-11)
    image32, _ = O.forward(plan, field, poses, samples=samples)
    np.testing.assert_allclose(image32, expected, rtol=5e-6, atol=5e-6)
    seed = np.linspace(-0.5, 0.8, image32.size)
    for arith, dtype, tol in ((O.ARITH_F32, O.F32, 5e-6), (O.ARITH_F64, O.F64, 5e-7)):
        volume, _, _ = O.vjp(plan, field, poses, seed.astype(np.float32 if dtype == O.F32 else np.float64),
                             samples=samples, flags=O.VJP_VOLUME, arith=arith, image_dtype=dtype)
        np.testing.assert_allclose(volume, matrix.T @ seed, rtol=tol, atol=tol / 10)


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_compensated_half_storage_matches_reference_fp32_marching_oracle(storage):
    """Reference test_projection_native_storage.py:41-84: FP32 marching and cell arithmetic
    on decoded half values (its oracle sums samples in FP64; the compensated sum matches it)."""
    grid, rays, data, samples = native_fixture()
    plan = plan_rays(grid, rays)
    bits = data[f"{storage}_bits"]
    code = O.F16 if storage == "float16" else O.BF16
    image, status = O.forward(plan, bits, IDENTITY, samples=samples, arith=O.ARITH_F32C, field_dtype=code,
                              image_dtype=O.F64)
    assert not status.any()
    np.testing.assert_allclose(image, data[f"{storage}_image"], rtol=1e-6, atol=1e-9)
    seed = np.asarray([1.5, -0.25, 3.0])
    volume, _, _ = O.vjp(plan, bits, IDENTITY, seed, samples=samples, flags=O.VJP_VOLUME, arith=O.ARITH_F32C,
                         field_dtype=code, image_dtype=O.F64)
    np.testing.assert_allclose(volume, data[f"{storage}_matrix"].T @ seed, rtol=2e-6, atol=1e-7)


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_fast_float32_half_storage_is_the_reference_fp32_marching_oracle(storage):
    """Reference test_projection_native_storage.py:41-84 is the fast_float32 arithmetic itself
    (FP32 marching, clamped FP32 weights, fused FP32 cell sum, FP64 ray sum): the FAST form
    reproduces its image to FP64 rounding and its weight matrix in the volume VJP."""
    grid, rays, data, samples = native_fixture()
    plan = plan_rays(grid, rays)
    bits = data[f"{storage}_bits"]
    code = O.F16 if storage == "float16" else O.BF16
    image, status = O.forward(plan, bits, IDENTITY, samples=samples, arith=O.ARITH_FAST, field_dtype=code,
                              image_dtype=O.F64)
    assert not status.any()
    np.testing.assert_allclose(image, data[f"{storage}_image"], rtol=1e-12, atol=1e-15)
    mixed, _ = O.forward(plan, bits, IDENTITY, samples=samples, arith=O.ARITH_MIXED, field_dtype=code,
                         image_dtype=O.F64)
    np.testing.assert_allclose(mixed, data[f"{storage}_image"], rtol=1e-6, atol=1e-9)
    seed = np.asarray([1.5, -0.25, 3.0])
    volume, _, _ = O.vjp(plan, bits, IDENTITY, seed, samples=samples, flags=O.VJP_VOLUME, arith=O.ARITH_FAST,
                         field_dtype=code, image_dtype=O.F64)
    np.testing.assert_allclose(volume, data[f"{storage}_matrix"].T @ seed, rtol=2e-6, atol=1e-7)


def test_analytic_ellipsoid_chords_under_sampling():
    """Sampled ellipsoids projected by the oracle approach the analytic chords (phantoms.py:57-97)."""
    facts = FACTS["ellipsoids"]
    grid = grid_from(facts["grid"])
    data = np.load(GOLDEN / "ellipsoids.npz")
    geometry = BatchedGeometry(tuple(panel_from(p) for p in facts["panels"]))
    plan = plan_rays(grid, geometry)
    poses = np.tile(IDENTITY, (len(geometry.views), 1))
    image, _ = O.forward(plan, data["values"], poses, samples=512, arith=O.ARITH_F64, image_dtype=O.F64)
    chords = data["chords"]
    hit = chords > 0.05
    assert hit.sum() > 30
    # voxel discretisation of a 0.75 mm grid: a few percent of the chord
    relative = np.abs(image[hit] - chords[hit]) / chords[hit]
    assert np.median(relative) < 0.03


def test_numpy_fp64_reference_rays():
    """Reference benchmarks/fullscan_guards.py:15-55 numpy FP64 rays at a non-identity pose."""
    from dpt_b200.geometry import ConeBeamIntrinsics

    facts = FACTS["guard"]
    grid = grid_from(facts["grid"])
    values = np.load(GOLDEN / "guard.npz")["values"]
    rays = np.load(GOLDEN / "guard.npz")["rays"]
    intrinsics = ConeBeamIntrinsics(200.0, 320.0, (10, 12), (2.0, 2.0))
    pose = np.asarray(facts["pose"])
    got = []
    for angle in facts["angles"]:
        plan = plan_rays(grid, intrinsics.view(angle))
        image, _ = O.forward(plan, values, pose, samples=facts["samples"], arith=O.ARITH_F64, image_dtype=O.F64)
        image = image.reshape(10, 12)
        got += [image[r, c] for r, c in facts["pixels"]]
    np.testing.assert_allclose(got, rays, rtol=1e-11, atol=1e-13)


def test_oracle_checks_flag_bad_field_and_pose():
    assert O.check_field(np.asarray([0.1, 0.0, 0.2], np.float32)) == 0
    assert O.check_field(np.asarray([0.1, -1e-9, 0.2], np.float32)) == 8
    assert O.check_field(np.asarray([0.1, np.nan], np.float32)) == 8
    assert O.check_pose(IDENTITY) == 0
    bad = IDENTITY.copy()
    bad[0] = -1.0  # reflection
    assert O.check_pose(bad) == 1
    skew = IDENTITY.copy()
    skew[1] = 1e-6
    assert O.check_pose(skew) == 1
    assert math.isfinite(float(IDENTITY.sum()))
