"""The CUDA deterministic adjoint gather against the oracle's all-ray gather (bit for bit) and
the reference's independent FP64 matrices, on the scenes of the reference's gather tests
(tests/python/warp_cpu/test_projection_adjoint_gather.py, test_projection_culled_adjoint.py):
the culled plan and the raw-pose call give the same bytes as the sum over all rays and
samples, repeatably; limits and diagnostics reject before any output is written."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from dpt_b200.contracts import ContractError, NumericalError
from dpt_b200.geometry import ConeBeamIntrinsics, RayBundleGeometry, RigidTransform
from dpt_b200.phantoms import centred_grid
from dpt_b200.projection import (
    ProjectionSpec,
    prepare_projection,
    prepare_projection_adjoint,
    project_optical_depth,
    projection_adjoint_gather,
    projection_vjp,
)
from dpt_b200.volumes import GridSpec
from oracle import oracle as O
from scenes import gather_matrix, gather_scene

pytestmark = pytest.mark.gpu
DEVICE = "cuda:0"
KINDS = ["culled_tilted", "culled_inside", "culled_negative_depth", "culled_underflow_plane",
         "culled_tolerated_rotation", "culled_bundle", "culled_large_tilted"]


def workspace_for(name, precision="float64"):
    grid, geometry, pose, samples = gather_scene(name)
    spec = ProjectionSpec(samples, active_pose=False, active_volume=True, precision=precision,
                          field_domain="signed_linear")
    ws = prepare_projection(grid, geometry, spec, device=DEVICE)
    return ws, grid, geometry, torch.tensor(pose, device=DEVICE), samples


@pytest.mark.parametrize("name", ["gather_nonsquare", "gather_bundle", "gather_clamped", "culled_tilted"])
def test_gather_matches_reference_matrix_oracle_and_is_repeatable(name):
    ws, grid, geometry, pose, samples = workspace_for(name)
    matrix = gather_matrix(name)
    plan = prepare_projection_adjoint(pose, workspace=ws)
    rng = np.random.default_rng(584291)
    for _ in range(5):
        seeds = rng.uniform(-1, 1, ws.plan.rays)
        cot = torch.tensor(seeds, device=DEVICE).reshape(ws.plan.image_shape)
        raw = projection_adjoint_gather(pose, cotangent=cot, workspace=ws)
        culled = projection_adjoint_gather(plan, cotangent=cot, workspace=ws)
        expected, _ = O.gather(ws.plan, pose.cpu().numpy(), seeds, samples=samples)
        assert raw.cpu().numpy().reshape(-1).tobytes() == expected.tobytes()
        assert culled.cpu().numpy().tobytes() == raw.cpu().numpy().tobytes()
        np.testing.assert_allclose(culled.cpu().numpy().reshape(-1), matrix.T @ seeds, rtol=2e-12, atol=2e-12)
        again = projection_adjoint_gather(plan, cotangent=cot, workspace=ws)
        assert again.cpu().numpy().tobytes() == culled.cpu().numpy().tobytes()


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_culled_gather_is_bitwise_the_all_ray_sum(kind, precision):
    ws, grid, geometry, pose, samples = workspace_for(kind)
    max_rays = 2048 if kind == "culled_large_tilted" else 256
    plan = prepare_projection_adjoint(pose, workspace=ws, max_rays_per_voxel=max_rays)
    rng = np.random.default_rng(754103)
    seeds = rng.normal(size=ws.plan.rays)
    seeds[::4] = 0.0
    cot = torch.tensor(seeds, device=DEVICE).reshape(ws.plan.image_shape)
    out_dtype = torch.float64 if precision == "float64" else torch.float32
    culled = torch.empty(grid.voxels, dtype=out_dtype, device=DEVICE)
    projection_adjoint_gather(plan, cotangent=cot, workspace=ws, out_mu=culled, volume_gradient_precision=precision)
    code = O.F64 if precision == "float64" else O.F32
    expected, status = O.gather(ws.plan, pose.cpu().numpy(), seeds, samples=samples, out_dtype=code)
    assert status == 0
    assert culled.cpu().numpy().tobytes() == expected.tobytes()
    raw = projection_adjoint_gather(pose, cotangent=cot, workspace=ws, volume_gradient_precision=precision,
                                    max_work=10**9)
    assert raw.cpu().numpy().reshape(-1).tobytes() == expected.tobytes()
    # accumulation adds the per-view sum to the existing values before the one rounding
    projection_adjoint_gather(plan, cotangent=cot, workspace=ws, out_mu=culled, volume_gradient_precision=precision,
                              accumulate=True)
    twice, _ = O.gather(ws.plan, pose.cpu().numpy(), seeds, samples=samples, out_dtype=code, out=expected,
                        accumulate=True)
    assert culled.cpu().numpy().tobytes() == twice.tobytes()
    assert plan.quadrature_nodes < grid.voxels * ws.plan.rays * samples
    if kind in ("culled_inside", "culled_underflow_plane"):
        assert plan.fallback_voxels > 0
    if kind == "culled_bundle":
        assert plan.candidate_rays == grid.voxels * ws.plan.rays


@pytest.mark.parametrize("shape", ["1x2x3", "1x3x2", "2x1x3", "3x1x2", "2x3x1", "3x2x1"])
def test_singleton_clamped_basis_is_conservatively_included(shape):
    ws, grid, geometry, pose, samples = workspace_for("singleton_" + shape)
    plan = prepare_projection_adjoint(pose, workspace=ws)
    seeds = np.array([(-1.0) ** i for i in range(ws.plan.rays)])
    cot = torch.tensor(seeds, device=DEVICE).reshape(ws.plan.image_shape)
    culled = projection_adjoint_gather(plan, cotangent=cot, workspace=ws)
    expected, _ = O.gather(ws.plan, pose.cpu().numpy(), seeds, samples=samples)
    assert culled.cpu().numpy().reshape(-1).tobytes() == expected.tobytes()


def test_multiview_scan_gathers_views_in_order_and_is_the_adjoint():
    grid = centred_grid((12, 10, 8), (1.0, 1.1, 0.9))
    geometry = ConeBeamIntrinsics(60.0, 100.0, (10, 12), (1.7, 1.6)).batch(
        tuple(2 * math.pi * k / 5 + 0.1 for k in range(5)))
    samples = 48
    ws = prepare_projection(grid, geometry, ProjectionSpec(samples, active_pose=False, active_volume=True,
                                                           precision="float64", field_domain="signed_linear"),
                            device=DEVICE)
    poses = torch.tensor(np.tile(RigidTransform().packed(), (5, 1)), device=DEVICE)
    plan = prepare_projection_adjoint(poses, workspace=ws, max_work=10**9, max_rays_per_voxel=4096)
    rng = np.random.default_rng(8)
    seeds = rng.normal(size=ws.plan.rays)
    cot = torch.tensor(seeds, device=DEVICE).reshape(ws.plan.image_shape)
    gathered = projection_adjoint_gather(plan, cotangent=cot, workspace=ws, max_work=10**9)
    expected, _ = O.gather(ws.plan, poses.cpu().numpy(), seeds, samples=samples)
    assert gathered.cpu().numpy().reshape(-1).tobytes() == expected.tobytes()
    values = torch.tensor(rng.normal(size=grid.shape).astype(np.float32), device=DEVICE)
    image = project_optical_depth(values, poses, workspace=ws)
    left = float((image.double() * cot).sum())
    right = float((values.double() * gathered).sum())
    assert abs(left - right) < 1e-11 * max(1.0, abs(left))
    scatter, _ = projection_vjp(values, poses, cotangent=cot, workspace=ws, pose_gradient=None,
                                volume_gradient_precision="float64")
    # the scatter VJP rounds each increment to FP32; the gather keeps every term in FP64
    np.testing.assert_allclose(scatter.cpu().numpy(), gathered.cpu().numpy(), rtol=2e-6,
                               atol=2e-6 * float(gathered.abs().max()))


def test_limits_and_bad_cotangents_reject_before_writing():
    ws, grid, geometry, pose, samples = workspace_for("gather_clamped")
    cot = torch.ones(ws.plan.image_shape, dtype=torch.float64, device=DEVICE)
    out = torch.full((grid.voxels,), 19.0, dtype=torch.float64, device=DEVICE)
    with pytest.raises(ContractError, match="max_work"):
        projection_adjoint_gather(pose, cotangent=cot, workspace=ws, out_mu=out, max_work=1)
    assert (out.cpu().numpy() == 19.0).all()
    with pytest.raises(NumericalError):
        projection_adjoint_gather(pose, cotangent=torch.full_like(cot, float("nan")), workspace=ws, out_mu=out)
    assert (out.cpu().numpy() == 19.0).all()
    ws2, *_ = workspace_for("culled_inside")
    pose2 = workspace_for("culled_inside")[3]
    for kwargs, message in [({"max_bytes": 1}, "max_bytes"), ({"max_prepare_voxels": 1}, "max_prepare_voxels"),
                            ({"max_work": 1}, "max_work"), ({"max_rays_per_voxel": 1}, "max_rays_per_voxel")]:
        with pytest.raises(ContractError, match=message):
            prepare_projection_adjoint(pose2, workspace=ws2, **kwargs)
    ws2.status.fill_(2)  # a pending diagnostic of an earlier call
    with pytest.raises(NumericalError):
        prepare_projection_adjoint(pose2, workspace=ws2)


def test_plan_belongs_to_its_workspace_and_rejects_aliases():
    ws, grid, geometry, pose, samples = workspace_for("culled_tilted")
    plan = prepare_projection_adjoint(pose, workspace=ws)
    other, *_ = workspace_for("culled_tilted")
    cot = torch.ones(ws.plan.image_shape, dtype=torch.float64, device=DEVICE)
    out = torch.full((grid.voxels,), 7.0, dtype=torch.float64, device=DEVICE)
    with pytest.raises(ContractError, match="original workspace configuration"):
        projection_adjoint_gather(plan, cotangent=cot, workspace=other, out_mu=out)
    assert (out.cpu().numpy() == 7.0).all()
    with pytest.raises(ContractError, match="overlaps prepared metrics"):
        projection_adjoint_gather(plan, cotangent=cot, workspace=ws, out_mu=plan.records[: grid.voxels])
    # the plan owns its rays: later changes to the pose buffer do not reach it
    first = projection_adjoint_gather(plan, cotangent=cot, workspace=ws)
    pose.fill_(float("nan"))
    second = projection_adjoint_gather(plan, cotangent=cot, workspace=ws)
    assert first.cpu().numpy().tobytes() == second.cpu().numpy().tobytes()
    ws.spec = ProjectionSpec(37, sampling_precision="float32", precision="float64")
    with pytest.raises(ContractError, match="strict float64"):
        projection_adjoint_gather(plan, cotangent=cot, workspace=ws)


def test_invalid_rays_and_overflowing_zero_weight_corners():
    grid = GridSpec((1, 1, 1), (1.0, 1.0, 1.0))
    tiny = RayBundleGeometry(((-2e-200, 0.0, 0.0),), ((2e-200, 0.0, 0.0),))
    ws = prepare_projection(grid, tiny, ProjectionSpec(3, precision="float64"), device=DEVICE)
    pose = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=DEVICE)
    with pytest.raises(NumericalError):
        prepare_projection_adjoint(pose, workspace=ws)
    grid = GridSpec((1, 1, 2), (10.0, 1.0, 1.0))
    ray = RayBundleGeometry(((-100.0, 0.0, 0.0),), ((0.0, 0.0, 0.0),))
    ws = prepare_projection(grid, ray, ProjectionSpec(1, precision="float64"), device=DEVICE)
    plan = prepare_projection_adjoint(pose, workspace=ws)
    seed = torch.tensor([1e308], dtype=torch.float64, device=DEVICE)
    for operator in (pose, plan):
        out = torch.empty(2, dtype=torch.float64, device=DEVICE)
        with pytest.raises(NumericalError):
            projection_adjoint_gather(operator, cotangent=seed, workspace=ws, out_mu=out)
        assert np.isnan(out.cpu().numpy()).all()


@pytest.mark.parametrize("name", ["gather_nonsquare", "gather_bundle", "gather_clamped"])
@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_cell_gauss_gather_matches_oracle_and_reference_exact_matrix(name, precision):
    grid, geometry, pose_np, _ = gather_scene(name)
    spec = ProjectionSpec(31, active_pose=False, active_volume=True, precision="float64",
                          integration="cell_gauss", field_domain="signed_linear")
    ws = prepare_projection(grid, geometry, spec, device=DEVICE)
    pose = torch.tensor(pose_np, device=DEVICE)
    matrix = np.load(__import__("scenes").GOLDEN / "gather.npz")[f"{name}_cells_matrix"]
    rng = np.random.default_rng(17)
    code = O.F64 if precision == "float64" else O.F32
    for _ in range(3):
        seeds = rng.uniform(-1, 1, ws.plan.rays)
        cot = torch.tensor(seeds, device=DEVICE).reshape(ws.plan.image_shape)
        out = projection_adjoint_gather(pose, cotangent=cot, workspace=ws, volume_gradient_precision=precision)
        expected, status = O.gather(ws.plan, pose_np, seeds, samples=31, cells=True, out_dtype=code)
        assert status == 0
        assert out.cpu().numpy().reshape(-1).tobytes() == expected.tobytes()
        if precision == "float64":
            np.testing.assert_allclose(out.cpu().numpy().reshape(-1), matrix.T @ seeds, rtol=2e-12, atol=2e-12)
    with pytest.raises(ContractError, match="strict float64 midpoint"):
        prepare_projection_adjoint(pose, workspace=ws)
