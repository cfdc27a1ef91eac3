"""The oracle on the small plain workload (64^3 at 1 mm, 8 cone views of 64^2 at 1.5 mm,
S = 128) against the reference's independent FP64 midpoint values of ``config1.npz``
(``make_config1_golden.py``): the whole image and the volume cotangent of the mean over
the central 32 x 32 pixels at seeded voxels.

Bars: FP64 images within 2e-11 (the reference's Projector contract, tests/python/warp_cpu/
test_projector_workflow.py:73-84); FP32 images within the reference's full-scan quality
contract for FP32 against FP64 (benchmarks/config/fullscan.json:85-91: relative L2 <= 1e-5,
RMSE <= 2e-5, max abs <= 5e-4; measured 1.2e-6, 1.6e-6, 9.7e-6 -- the Projector contract's
elementwise 5e-6 was set on a 3x3x4 grid and a few of these 128-sample rays exceed it).  The
VJP of the central mean meets the Projector contract's rtol 5e-6 / atol 5e-7 and, tighter,
2e-5 (FP32) or 1e-8 (FP64, whose increments the reference rounds to FP32 before they are
summed) of its largest value; the FP32 pair (image, cotangent) satisfies the adjoint identity
of the full-scan contract (fullscan.json:99-103, 2e-5).
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from dpt_b200.plan import plan_rays
from oracle import oracle as O
from scenes import GOLDEN, config1_scene, identity_poses


@pytest.fixture(scope="module")
def scene():
    grid, geometry, values = config1_scene()
    golden = np.load(GOLDEN / "config1.npz")
    return grid, geometry, values, golden


def central_mean_cotangent(views: int, rows: int, cols: int, central: int, dtype) -> np.ndarray:
    cot = np.zeros((views, rows, cols), dtype=dtype)
    r0, c0 = (rows - central) // 2, (cols - central) // 2
    cot[:, r0:r0 + central, c0:c0 + central] = 1.0 / (views * central * central)
    return cot


def test_phantom_is_the_one_the_fixture_was_made_from(scene):
    _, _, values, golden = scene
    digest = hashlib.sha256(np.ascontiguousarray(values, dtype=np.float32).tobytes()).hexdigest()
    assert digest == golden["field_sha256"].item().decode()


@pytest.mark.parametrize("arith", [O.ARITH_F32, O.ARITH_F64])
def test_oracle_image_and_vjp_match_reference_values(scene, arith):
    grid, geometry, values, golden = scene
    plan = plan_rays(grid, geometry)
    views = len(geometry.views)
    poses = identity_poses(views)
    samples = int(golden["samples"])
    wide = arith == O.ARITH_F64
    image, status = O.forward(plan, values, poses, samples=samples, arith=arith,
                              image_dtype=O.F64 if wide else O.F32)
    assert not status.any()
    expected = golden["image"].reshape(-1)
    if wide:
        np.testing.assert_allclose(image, expected, rtol=2e-11, atol=2e-11)
    else:
        error = image.astype(np.float64) - expected
        assert np.linalg.norm(error) <= 1e-5 * np.linalg.norm(expected)
        assert np.sqrt(np.mean(error * error)) <= 2e-5
        assert np.abs(error).max() <= 5e-4

    rows, cols = geometry.shape_rows_columns
    cot = central_mean_cotangent(views, rows, cols, int(golden["central"]), np.float64 if wide else np.float32)
    volume, _, status = O.vjp(plan, values, poses, cot, samples=samples, flags=O.VJP_VOLUME, arith=arith,
                              image_dtype=O.F64 if wide else O.F32)
    assert not status.any()
    reference = golden["vjp_values"]
    got = volume[golden["vjp_voxels"]]
    scale = np.abs(reference).max()
    assert scale > 0
    np.testing.assert_allclose(got, reference, rtol=5e-6, atol=5e-7)
    np.testing.assert_allclose(got, reference, rtol=0, atol=(1e-8 if wide else 2e-5) * scale)
    if not wide:
        lhs = float(np.dot(image.astype(np.float64), cot.reshape(-1).astype(np.float64)))
        rhs = float(np.dot(values.reshape(-1).astype(np.float64), volume))
        assert abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-300) <= 2e-5
