"""The small plain workload on the GPU through the public ``Projector``: 64^3 at 1 mm,
seeded ellipsoid phantom, 8 cone views over 360 deg (SOD 500, SDD 1000), 64 x 64 detector at
1.5 mm, S = 128; loss = mean over the central 32 x 32 detector pixels of every view.

Against the oracle on the same inputs: images and per-ray clip intervals and realised counts
bit for bit, the volume gradient within 2e-6 relative L2 (FP32 atomic order and the FP32
field gradient), the per-view
pose gradient within 1e-9 (FP64 reduction order).  Against the reference's independent FP64
midpoint values (``config1.npz``): FP64 images within the reference Projector contract's
2e-11 (tests/python/warp_cpu/test_projector_workflow.py:73-84), FP32 images within the
full-scan quality contract for FP32 against FP64 (benchmarks/config/fullscan.json:85-91:
relative L2 1e-5, RMSE 2e-5, max abs 5e-4), the central-mean gradient at the fixture's voxels
within the Projector contract's rtol 5e-6 / atol 5e-7 and within 2e-5 (FP32) or 1e-7 (FP64:
increments rounded to FP32 as the reference rounds them, and the FP32 field's gradient is
FP32) of its largest value, and the adjoint
identity of the full-scan contract (2e-5).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from dpt_b200.torch import Projector
from dpt_b200.torch import _projection_ops as ops
from oracle import oracle as O
from scenes import GOLDEN, config1_scene, identity_poses

pytestmark = pytest.mark.gpu
DEVICE = "cuda:0"


def rel_l2(a, b) -> float:
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_config1_projector_matches_oracle_and_reference_values(precision):
    grid, geometry, values = config1_scene()
    golden = np.load(GOLDEN / "config1.npz")
    samples, central = int(golden["samples"]), int(golden["central"])
    views = len(geometry.views)
    rows, cols = geometry.shape_rows_columns
    wide = precision == "fp64"
    arith, image_dtype = (O.ARITH_F64, O.F64) if wide else (O.ARITH_F32, O.F32)

    module = Projector(grid=grid, geometry=geometry, precision=precision, samples_per_ray=samples)
    field = torch.tensor(values, device=DEVICE, requires_grad=True)
    tangent = torch.zeros((views, 6), dtype=torch.float64, device=DEVICE, requires_grad=True)
    image = module(field, tangent)
    r0, c0 = (rows - central) // 2, (cols - central) // 2
    loss = image[:, r0:r0 + central, c0:c0 + central].mean()
    loss.backward()
    torch.cuda.synchronize()

    ws = ops.workspace(field.detach(), module.configuration, True, True)
    poses = identity_poses(views)
    got_image = image.detach().cpu().numpy().reshape(-1)
    expected, status = O.forward(ws.plan, values, poses, samples=samples, arith=arith, image_dtype=image_dtype)
    assert not status.any()
    np.testing.assert_array_equal(got_image, expected)
    lower, upper, realised = (t.cpu().numpy() for t in ws.counts(torch.tensor(poses, device=DEVICE)))
    e_lower, e_upper, e_realised = O.counts(ws.plan, poses, samples=samples, arith=arith)
    np.testing.assert_array_equal(lower, e_lower)
    np.testing.assert_array_equal(upper, e_upper)
    np.testing.assert_array_equal(realised, e_realised)
    reference_image = golden["image"].reshape(-1)
    if wide:
        np.testing.assert_allclose(got_image, reference_image, rtol=2e-11, atol=2e-11)
    else:
        error = got_image.astype(np.float64) - reference_image
        assert np.linalg.norm(error) <= 1e-5 * np.linalg.norm(reference_image)
        assert np.sqrt(np.mean(error * error)) <= 2e-5
        assert np.abs(error).max() <= 5e-4

    cot = np.zeros((views, rows, cols), dtype=np.float64 if wide else np.float32)
    cot[:, r0:r0 + central, c0:c0 + central] = 1.0 / (views * central * central)
    e_volume, e_pose12, status = O.vjp(ws.plan, values, poses, cot, samples=samples,
                                       flags=O.VJP_VOLUME | O.VJP_POSE6, arith=arith, image_dtype=image_dtype)
    assert not status.any()
    volume = field.grad.detach().cpu().numpy().reshape(-1).astype(np.float64)
    assert rel_l2(volume, e_volume) < 2e-6
    # tangent gradient of an identity anchor: the local-right 6-vector of the kernel
    np.testing.assert_allclose(tangent.grad.cpu().numpy(), e_pose12, rtol=1e-9, atol=1e-15)

    reference = golden["vjp_values"]
    scale = np.abs(reference).max()
    np.testing.assert_allclose(volume[golden["vjp_voxels"]], reference, rtol=5e-6, atol=5e-7)
    np.testing.assert_allclose(volume[golden["vjp_voxels"]], reference, rtol=0,
                               atol=(1e-7 if wide else 2e-5) * scale)
    lhs = float(np.dot(got_image.astype(np.float64), cot.reshape(-1).astype(np.float64)))
    rhs = float(np.dot(values.reshape(-1).astype(np.float64), volume))
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-300) <= 2e-5
