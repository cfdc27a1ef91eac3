"""CUDA kernels (through the C ABI) against the CPU oracle on the same seeded inputs.

Bars: forward images, clip intervals and realised sample counts are bit-exact for
the FP32 and FP64 arithmetic (same floating-point contract); FP32 volume
gradients agree to 2e-5 relative L2 (atomic summation order), pose gradients to
1e-9 relative (FP64 reduction order); the compensated form agrees to 1e-6.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from dpt_b200 import _native as N
from dpt_b200.plan import plan_rays
from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace
from oracle import oracle as O
from scenes import cone_scene, fp32_fixture, identity_poses, mixed_panels, poses_for

pytestmark = pytest.mark.gpu

ARITH = {"float32": O.ARITH_F32, "float64": O.ARITH_F64, "compensated": O.ARITH_F32C,
         "mixed_float32": O.ARITH_MIXED, "fast_float32": O.ARITH_FAST, "cell_gauss": O.ARITH_CELLS}


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def workspace(grid, geometry, samples, sampling="float32", precision="float32", storage="float32",
              layout="replicated", widen=None, active_pose=True, domain="physical"):
    integration = "midpoint"
    if sampling == "cell_gauss":
        sampling, integration = "float64", "cell_gauss"
    spec = ProjectionSpec(samples, precision=precision, sampling_precision=sampling,
                          storage_precision=storage, layout=layout, widen_views=widen,
                          integration=integration, active_pose=active_pose, field_domain=domain)
    return ProjectionWorkspace(plan_rays(grid, geometry), spec, "cuda:0")


def device_inputs(values, poses, dtype=torch.float32):
    field = torch.tensor(np.asarray(values, dtype=np.float32), device="cuda:0").to(dtype).contiguous()
    return field, torch.tensor(poses, dtype=torch.float64, device="cuda:0")


@pytest.mark.parametrize("samples", [17, 97, 1024])
def test_fp32_forward_bit_exact_on_reference_matrix_scene(samples):
    grid, rays, data = fp32_fixture()
    ws = workspace(grid, rays, samples)
    field, pose = device_inputs(data["values"].reshape(grid.shape), data["pose"])
    image = ws.forward(field, pose).cpu().numpy()
    expected, status = O.forward(ws.plan, data["values"], data["pose"], samples=samples)
    assert not status.any()
    np.testing.assert_array_equal(image, expected)
    # and within the reference test's tolerance of its own FP32 weight matrix
    np.testing.assert_allclose(image, data[f"matrix_{samples}"] @ data["values"].astype(np.float64),
                               rtol=2e-5, atol=3e-7)


@pytest.mark.parametrize("sampling", ["float32", "float64", "compensated"])
@pytest.mark.parametrize("layout", ["replicated", "direct"])
def test_cone_forward_and_counts_bit_exact(sampling, layout):
    grid, geometry, values = cone_scene()
    poses = poses_for(len(geometry.views))
    precision = "float64" if sampling == "float64" else "float32"
    ws = workspace(grid, geometry, 61, sampling, precision, layout=layout)
    field, pose = device_inputs(values, poses)
    image = ws.forward(field, pose).cpu().numpy().reshape(-1)
    expected, status = O.forward(ws.plan, values, poses, samples=61, arith=ARITH[sampling],
                                 image_dtype=O.F64 if precision == "float64" else O.F32)
    assert not status.any()
    np.testing.assert_array_equal(image, expected)
    lower, upper, realised = (t.cpu().numpy() for t in ws.counts(pose))
    e_lower, e_upper, e_realised = O.counts(ws.plan, poses, samples=61, arith=ARITH[sampling])
    np.testing.assert_array_equal(lower, e_lower)
    np.testing.assert_array_equal(upper, e_upper)
    np.testing.assert_array_equal(realised, e_realised)
    assert realised.sum() > 0


def test_parallel_and_curved_panels_match_oracle():
    grid, _, values = cone_scene()
    geometry = mixed_panels(grid)
    poses = poses_for(3, seed=4)
    ws = workspace(grid, geometry, 45)
    field, pose = device_inputs(values, poses)
    image = ws.forward(field, pose).cpu().numpy().reshape(-1)
    expected, _ = O.forward(ws.plan, values, poses, samples=45)
    # curved panels use the device's sincos: compare with a tolerance there
    np.testing.assert_array_equal(image[: 2 * 99], expected[: 2 * 99])
    np.testing.assert_allclose(image[2 * 99:], expected[2 * 99:], rtol=1e-5, atol=1e-7)
    assert np.abs(expected).sum() > 0


@pytest.mark.parametrize("sampling", ["float32", "float64", "compensated"])
@pytest.mark.parametrize("pose_form", ["matrix", "tangent"])
def test_joint_vjp_matches_oracle(sampling, pose_form):
    grid, geometry, values = cone_scene()
    views = len(geometry.views)
    poses = poses_for(views, seed=2)
    precision = "float64" if sampling == "float64" else "float32"
    ws = workspace(grid, geometry, 53, sampling, precision, widen=3)
    field, pose = device_inputs(values, poses)
    rng = np.random.default_rng(9)
    seed = rng.uniform(-1.0, 1.0, ws.plan.rays).astype(np.float64 if precision == "float64" else np.float32)
    cot = torch.tensor(seed, device="cuda:0").reshape(ws.plan.image_shape)
    volume, pose_grad = ws.vjp(field, pose, cot, volume=True, pose=pose_form)
    flags = O.VJP_VOLUME | (O.VJP_POSE12 if pose_form == "matrix" else O.VJP_POSE6)
    e_volume, e_pose, status = O.vjp(ws.plan, values, poses, seed, samples=53, flags=flags,
                                     arith=ARITH[sampling], image_dtype=O.F64 if precision == "float64" else O.F32)
    assert not status.any()
    assert rel_l2(volume.cpu().numpy().reshape(-1), e_volume) < 2e-6
    np.testing.assert_allclose(pose_grad.cpu().numpy(), e_pose, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_half_storage_forward_and_vjp_match_oracle(storage):
    grid, geometry, values = cone_scene()
    poses = poses_for(len(geometry.views), seed=3)
    ws = workspace(grid, geometry, 47, "compensated", storage=storage)
    dtype = torch.float16 if storage == "float16" else torch.bfloat16
    field, pose = device_inputs(values, poses, dtype)
    half = field.cpu()
    image = ws.forward(field, pose).cpu().numpy().reshape(-1)
    code = O.F16 if storage == "float16" else O.BF16
    raw = half.view(torch.int16).numpy().view(np.uint16)
    expected, _ = O.forward(ws.plan, raw, poses, samples=47, arith=O.ARITH_F32C, field_dtype=code)
    np.testing.assert_array_equal(image, expected)
    seed = np.random.default_rng(1).uniform(0.1, 1.0, ws.plan.rays).astype(np.float32)
    cot = torch.tensor(seed, device="cuda:0").reshape(ws.plan.image_shape)
    volume, pose_grad = ws.vjp(field, pose, cot, volume=True, pose="tangent")
    e_volume, e_pose, _ = O.vjp(ws.plan, raw, poses, seed, samples=47, flags=O.VJP_VOLUME | O.VJP_POSE6,
                                arith=O.ARITH_F32C, field_dtype=code)
    assert rel_l2(volume.cpu().numpy().reshape(-1), e_volume) < 2e-6
    np.testing.assert_allclose(pose_grad.cpu().numpy(), e_pose, rtol=1e-9, atol=1e-12)


def test_per_ray_pose_rows_sum_to_view_gradient():
    grid, geometry, values = cone_scene(views=2)
    poses = poses_for(2, seed=6)
    ws = workspace(grid, geometry, 40)
    field, pose = device_inputs(values, poses)
    seed = np.random.default_rng(2).uniform(-1, 1, ws.plan.rays).astype(np.float32)
    cot = torch.tensor(seed, device="cuda:0").reshape(ws.plan.image_shape)
    rows = ws.pose_sensitivities(field, pose, cot).cpu().numpy()
    _, tangent = ws.vjp(field, pose, cot, volume=False, pose="tangent")
    per_view = rows.reshape(2, -1, 6).sum(axis=1)
    np.testing.assert_allclose(per_view, tangent.cpu().numpy(), rtol=1e-10, atol=1e-13)
    _, e_rows, _ = O.vjp(ws.plan, values, poses, seed, samples=40, flags=O.VJP_PER_RAY6)
    np.testing.assert_array_equal(rows, e_rows)


def test_identity_pose_bundle_single_voxel_known_answer():
    """Clipped single-voxel case of the reference FP32 tests: L = 0.025*0.7."""
    from dpt_b200.geometry import RayBundleGeometry
    from dpt_b200.volumes import GridSpec

    grid = GridSpec((1, 1, 1), (1.0, 1.0, 1.0))
    rays = RayBundleGeometry(((-2.0, 0.0, 0.0),), ((0.2, 0.0, 0.0),))
    ws = workspace(grid, rays, 1024)
    field, pose = device_inputs(np.array([[[0.025]]], dtype=np.float32), identity_poses(1))
    image = ws.forward(field, pose).cpu().numpy()
    np.testing.assert_allclose(image, [0.025 * 0.7], rtol=2e-5)
    cot = torch.ones(1, device="cuda:0")
    volume, tangent = ws.vjp(field, pose, cot, volume=True, pose="tangent")
    np.testing.assert_allclose(volume.cpu().numpy().reshape(-1), [0.7], rtol=2e-5)
    np.testing.assert_allclose(tangent.cpu().numpy().reshape(-1), [-0.025, 0, 0, 0, 0, 0], rtol=2e-5, atol=1e-8)


@pytest.mark.parametrize("block_cols", [8, 32, 64])
def test_block_tile_shape_changes_no_result(block_cols):
    grid, geometry, values = cone_scene(detector=(37, 45))
    poses = poses_for(len(geometry.views), seed=11)
    field, pose = device_inputs(values, poses)
    base = workspace(grid, geometry, 29)
    spec = ProjectionSpec(29, sampling_precision="float32", block_cols=block_cols)
    tuned = ProjectionWorkspace(plan_rays(grid, geometry), spec, "cuda:0")
    torch.testing.assert_close(tuned.forward(field, pose), base.forward(field, pose), rtol=0, atol=0)
    cot = torch.rand(base.plan.image_shape, device="cuda:0")
    v0, p0 = base.vjp(field, pose, cot, volume=True, pose="matrix")
    v1, p1 = tuned.vjp(field, pose, cot, volume=True, pose="matrix")
    assert rel_l2(v1.cpu().numpy(), v0.cpu().numpy()) < 1e-6
    torch.testing.assert_close(p1, p0, rtol=1e-10, atol=1e-13)


# ---------------------------------------------------- reference sampling options

@pytest.mark.parametrize("sampling", ["mixed_float32", "fast_float32", "cell_gauss"])
@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_reference_sampling_options_forward_and_counts_bit_exact(sampling, precision):
    grid, geometry, values = cone_scene()
    poses = poses_for(len(geometry.views), seed=5)
    ws = workspace(grid, geometry, 61, sampling, precision, active_pose=sampling == "cell_gauss")
    field, pose = device_inputs(values, poses)
    image = ws.forward(field, pose).cpu().numpy().reshape(-1)
    expected, status = O.forward(ws.plan, values, poses, samples=61, arith=ARITH[sampling],
                                 image_dtype=O.F64 if precision == "float64" else O.F32)
    assert not status.any()
    np.testing.assert_array_equal(image, expected)
    lower, upper, realised = (t.cpu().numpy() for t in ws.counts(pose))
    e_lower, e_upper, e_realised = O.counts(ws.plan, poses, samples=61, arith=ARITH[sampling])
    np.testing.assert_array_equal(lower, e_lower)
    np.testing.assert_array_equal(upper, e_upper)
    np.testing.assert_array_equal(realised, e_realised)


@pytest.mark.parametrize("sampling", ["mixed_float32", "fast_float32"])
def test_fixed_pose_samplings_volume_vjp_match_oracle(sampling):
    grid, geometry, values = cone_scene()
    poses = poses_for(len(geometry.views), seed=6)
    ws = workspace(grid, geometry, 53, sampling, "float64", active_pose=False, widen=3)
    field, pose = device_inputs(values, poses)
    seed = np.random.default_rng(4).uniform(-1.0, 1.0, ws.plan.rays)
    cot = torch.tensor(seed, device="cuda:0").reshape(ws.plan.image_shape)
    volume, _ = ws.vjp(field, pose, cot, volume=True, pose=None)
    e_volume, _, status = O.vjp(ws.plan, values, poses, seed, samples=53, flags=O.VJP_VOLUME,
                                arith=ARITH[sampling], image_dtype=O.F64)
    assert not status.any()
    assert rel_l2(volume.cpu().numpy().reshape(-1), e_volume) < 2e-6
    with pytest.raises(Exception):
        ws.vjp(field, pose, cot, volume=False, pose="tangent")


@pytest.mark.parametrize("pose_form", ["matrix", "tangent"])
def test_cell_gauss_joint_vjp_matches_oracle(pose_form):
    grid, geometry, values = cone_scene()
    poses = poses_for(len(geometry.views), seed=7)
    ws = workspace(grid, geometry, 1, "cell_gauss", "float64", widen=2)
    field, pose = device_inputs(values, poses)
    seed = np.random.default_rng(8).uniform(-1.0, 1.0, ws.plan.rays)
    cot = torch.tensor(seed, device="cuda:0").reshape(ws.plan.image_shape)
    volume, pose_grad = ws.vjp(field, pose, cot, volume=True, pose=pose_form)
    flags = O.VJP_VOLUME | (O.VJP_POSE12 if pose_form == "matrix" else O.VJP_POSE6)
    e_volume, e_pose, status = O.vjp(ws.plan, values, poses, seed, samples=1, flags=flags,
                                     arith=O.ARITH_CELLS, image_dtype=O.F64)
    assert not status.any()
    assert rel_l2(volume.cpu().numpy().reshape(-1), e_volume) < 2e-6
    np.testing.assert_allclose(pose_grad.cpu().numpy(), e_pose, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
@pytest.mark.parametrize("sampling", ["float64", "fast_float32", "cell_gauss"])
def test_half_storage_under_reference_samplings_matches_oracle(storage, sampling):
    grid, geometry, values = cone_scene()
    poses = poses_for(len(geometry.views), seed=9)
    ws = workspace(grid, geometry, 47, sampling, "float64", storage=storage,
                   active_pose=sampling != "fast_float32")
    dtype = torch.float16 if storage == "float16" else torch.bfloat16
    field, pose = device_inputs(values, poses, dtype)
    raw = field.cpu().view(torch.int16).numpy().view(np.uint16)
    code = O.F16 if storage == "float16" else O.BF16
    image = ws.forward(field, pose).cpu().numpy().reshape(-1)
    expected, _ = O.forward(ws.plan, raw, poses, samples=47, arith=ARITH[sampling], field_dtype=code,
                            image_dtype=O.F64)
    np.testing.assert_array_equal(image, expected)


def test_signed_linear_domain_accepts_negative_fields():
    from dpt_b200.contracts import TrialDomainError

    grid, geometry, values = cone_scene()
    poses = poses_for(len(geometry.views), seed=10)
    signed = values - 0.5 * values.max()
    field, pose = device_inputs(signed, poses)
    ws = workspace(grid, geometry, 33, "float64", "float64", domain="signed_linear")
    image = ws.forward(field, pose).cpu().numpy().reshape(-1)
    expected, _ = O.forward(ws.plan, signed, poses, samples=33, arith=O.ARITH_F64, image_dtype=O.F64)
    np.testing.assert_array_equal(image, expected)
    assert (image < 0).any()
    physical = workspace(grid, geometry, 33, "float64", "float64")
    with pytest.raises(TrialDomainError):
        physical.forward(field, pose)


@pytest.mark.parametrize("pose_form", ["matrix", "tangent"])
@pytest.mark.parametrize("volume", [True, False])
@pytest.mark.parametrize("sampling,storage", [("float32", "float32"), ("compensated", "bfloat16")])
@pytest.mark.parametrize("shape", [(14, 16, 18), (12, 16, 32)])  # the second: power-of-two nx, ny
def test_split_pose_vjp_from_forward_moments_equals_joint_vjp(pose_form, volume, sampling, storage, shape):
    """A forward that stores the pose moments writes the same image, and the VJP that then
    forms the pose gradient from them (no second sampling pass) equals the joint VJP."""
    grid, geometry, values = cone_scene(shape=shape)
    poses = poses_for(len(geometry.views), seed=12)
    dtype = torch.bfloat16 if storage == "bfloat16" else torch.float32
    field, pose = device_inputs(values, poses, dtype)
    joint = workspace(grid, geometry, 53, sampling, storage=storage, widen=3)
    split = workspace(grid, geometry, 53, sampling, storage=storage, widen=3)
    image = joint.forward(field, pose)
    image_m = split.forward(field, pose, moments=True)
    torch.testing.assert_close(image_m, image, rtol=0, atol=0)
    cot = torch.rand(image.shape, device="cuda:0") - 0.5
    v0, p0 = joint.vjp(field, pose, cot, volume=volume, pose=pose_form)
    v1, p1 = split.vjp(field, pose, cot, volume=volume, pose=pose_form)
    torch.testing.assert_close(p1, p0, rtol=0, atol=0)
    if volume:
        assert rel_l2(v1.cpu().numpy(), v0.cpu().numpy()) < 1e-6
    # the moments are consumed: a second VJP samples again and still agrees
    _, p2 = split.vjp(field, pose, cot, volume=False, pose=pose_form)
    torch.testing.assert_close(p2, p0, rtol=0, atol=0)
    # changed poses after the forward: the stored moments are not used
    pose.add_(0.0)
    split.forward(field, pose, moments=True)
    pose.mul_(1.0)  # bumps the version counter
    _, p3 = split.vjp(field, pose, cot, volume=False, pose=pose_form)
    torch.testing.assert_close(p3, p0, rtol=0, atol=0)


@pytest.mark.parametrize("samples", [5, 9])
def test_compensated_sparse_samples_take_per_sample_form(samples):
    """Samples more than one cell plane apart take the per-sample form on both sides: the
    forward agrees bit for bit with the oracle, the joint VJP to the tolerances above, and
    both stay within the compensated form's error of the FP64 path."""
    grid, geometry, values = cone_scene()
    views = len(geometry.views)
    poses = poses_for(views, seed=3)
    ws = workspace(grid, geometry, samples, "compensated", widen=3)
    field, pose = device_inputs(values, poses)
    image = ws.forward(field, pose).cpu().numpy().reshape(-1)
    expected, status = O.forward(ws.plan, values, poses, samples=samples, arith=O.ARITH_F32C)
    assert not status.any()
    np.testing.assert_array_equal(image, expected)
    exact, _ = O.forward(ws.plan, values, poses, samples=samples, arith=O.ARITH_F64, image_dtype=O.F64)
    assert rel_l2(image, exact) < 1e-6
    rng = np.random.default_rng(11)
    seed = rng.uniform(-1.0, 1.0, ws.plan.rays).astype(np.float32)
    cot = torch.tensor(seed, device="cuda:0").reshape(ws.plan.image_shape)
    volume, pose_grad = ws.vjp(field, pose, cot, volume=True, pose="tangent")
    e_volume, e_pose, status = O.vjp(ws.plan, values, poses, seed, samples=samples,
                                     flags=O.VJP_VOLUME | O.VJP_POSE6, arith=O.ARITH_F32C)
    assert not status.any()
    assert rel_l2(volume.cpu().numpy().reshape(-1), e_volume) < 2e-6
    np.testing.assert_allclose(pose_grad.cpu().numpy(), e_pose, rtol=1e-9, atol=1e-12)
