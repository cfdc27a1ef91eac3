"""Pose recovery on the head workload: 512x507x76 anisotropic grid (0.45x0.45x2.5 mm,
direction cosines rotated 15 deg about z), AP and lateral 256x256 views, 768 samples.

Checks: FP64 central differences of the L2 loss against the autograd pose gradient on all
6 DoF (translation step 1e-3 mm, rotation step 1e-7 rad) and against the volume gradient
on 64 random voxels; 120 first-order iterations through the autograd path reduce the pose
error; Gauss-Newton with the per-ray pose Jacobian recovers the seeded ground-truth pose.

The rotation step is small because the loss is only piecewise smooth: the trilinear field
has slope jumps on every cell face, and the phantom's per-voxel brain noise and voxelised
bone edges make them large.  A 1e-3 rad turn moves the periphery ~0.1 mm, across many
faces, and central differences there miss the derivative by up to 20%; at 1e-7 rad
(<= 2e-5 mm of motion) they agree with it to 0.05%.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from dpt_b200.geometry import RigidTransform
from dpt_b200.imaging import standard_views
from dpt_b200.phantoms import centred_grid, head_phantom
from dpt_b200.plan import plan_rays
from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace
from dpt_b200.torch import Projector, compose_pose

pytestmark = pytest.mark.gpu
DEVICE = "cuda:0"


@pytest.fixture(scope="module")
def head():
    angle = math.radians(15.0)
    c, s = math.cos(angle), math.sin(angle)
    grid = centred_grid((76, 507, 512), (0.45, 0.45, 2.5), (c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0))
    values = head_phantom(grid, seed=4)
    geometry = standard_views(grid, ("ap", "lateral"), shape=(256, 256))
    rng = np.random.default_rng(2024)
    truth = np.concatenate([rng.uniform(-10.0, 10.0, 3), np.radians(rng.uniform(-5.0, 5.0, 3))])
    return grid, geometry, torch.tensor(values, device=DEVICE), torch.tensor(truth, device=DEVICE)


def _loss(module, field, tangent, target):
    image = module(field, tangent)
    residual = image.double() - target
    return 0.5 * (residual * residual).sum()


def test_fp64_finite_differences_pose_and_volume(head):
    grid, geometry, field, truth = head
    module = Projector(grid=grid, geometry=geometry, precision="fp64", samples_per_ray=768)
    with torch.no_grad():
        target = module(field, truth).double()
    start = torch.zeros(6, dtype=torch.float64, device=DEVICE)
    tangent = start.clone().requires_grad_(True)
    volume = field.clone().requires_grad_(True)
    loss = _loss(module, volume, tangent, target)
    pose_gradient, volume_gradient = torch.autograd.grad(loss, (tangent, volume))
    with torch.no_grad():
        for k in range(6):
            h = 1e-3 if k < 3 else 1e-7
            step = torch.zeros(6, dtype=torch.float64, device=DEVICE)
            step[k] = h
            fd = (_loss(module, field, start + step, target) - _loss(module, field, start - step, target)) / (2 * h)
            analytic = pose_gradient[k]
            assert abs(float(fd - analytic)) <= 1e-7 * float(pose_gradient.abs().max()) + 0.005 * abs(float(analytic)), (k, float(fd), float(analytic))
        rng = np.random.default_rng(7)
        flat = field.reshape(-1)
        # voxels with tissue (the field must stay non-negative under the central step)
        touched = torch.nonzero((volume_gradient.reshape(-1).abs() > 0) & (flat > 1e-3)).reshape(-1).cpu().numpy()
        for voxel in rng.choice(touched, 64, replace=False):
            value = float(flat[voxel])
            delta = 1e-3 * value
            plus, minus = flat.clone(), flat.clone()
            plus[voxel] = value + delta
            # the field must stay non-negative: air voxels take a one-sided difference
            # (the loss is quadratic in one voxel, so the secant slope is exact at the
            # midpoint and within curvature * delta / 2 of the slope at the voxel value)
            minus[voxel] = max(value - delta, 0.0)
            lp = _loss(module, plus.reshape(field.shape), start, target)
            lm = _loss(module, minus.reshape(field.shape), start, target)
            # plus/minus are rounded to FP32 storage: use the realised step
            realised = float(plus[voxel]) - float(minus[voxel])
            fd = float(lp - lm) / realised
            analytic = float(volume_gradient.reshape(-1)[voxel])
            assert abs(fd - analytic) <= 2e-3 * abs(analytic) + 1e-9, (int(voxel), fd, analytic)


def test_first_order_iterations_reduce_the_pose_error(head):
    grid, geometry, field, truth = head
    module = Projector(grid=grid, geometry=geometry, precision="fp32", samples_per_ray=768)
    with torch.no_grad():
        target = module(field, truth).double()
    tangent = torch.zeros(6, dtype=torch.float64, device=DEVICE, requires_grad=True)
    optimiser = torch.optim.Adam([tangent], lr=0.5, betas=(0.8, 0.95))
    scale = torch.tensor([1.0, 1.0, 1.0, 0.01, 0.01, 0.01], dtype=torch.float64, device=DEVICE)
    losses = []
    for iteration in range(120):
        optimiser.zero_grad()
        loss = _loss(module, field, tangent * scale, target)
        loss.backward()
        optimiser.step()
        losses.append(float(loss))
        if iteration == 60:
            for group in optimiser.param_groups:
                group["lr"] = 0.1
    final = (tangent.detach() * scale - truth).abs()
    initial = truth.abs()
    assert losses[-1] < 0.05 * losses[0]
    assert float(final[:3].max()) < 0.25 * float(initial[:3].max())
    assert float(final[3:].max()) < 0.25 * float(initial[3:].max())


def test_gauss_newton_with_per_ray_jacobian_recovers_the_pose(head):
    grid, geometry, field, truth = head
    views = len(geometry.views)
    workspace = ProjectionWorkspace(plan_rays(grid, geometry), ProjectionSpec(768, sampling_precision="float32"),
                                    DEVICE)
    anchor = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=DEVICE)

    def poses(xi):
        return compose_pose(anchor, xi).expand(views, 12).contiguous()

    target = workspace.forward(field, poses(truth)).double()
    ones = torch.ones(workspace.plan.image_shape, dtype=torch.float32, device=DEVICE)
    xi = torch.zeros(6, dtype=torch.float64, device=DEVICE)
    for _ in range(25):
        residual = (workspace.forward(field, poses(xi)).double() - target).reshape(-1)
        rows = workspace.pose_sensitivities(field, poses(xi), ones)  # local-right rows at xi
        normal = rows.T @ rows + 1e-9 * torch.eye(6, dtype=torch.float64, device=DEVICE)
        delta = -torch.linalg.solve(normal, rows.T @ residual)
        # local-right increment: compose on the right, then express as chart coordinates
        updated = compose_pose(compose_pose(anchor, xi), delta)
        xi = _chart(updated)
        if float(delta.abs().max()) < 1e-7:
            break
    error = (xi - truth).abs()
    assert float(error[:3].max()) < 0.01  # mm
    assert float(error[3:].max()) < 1e-4  # rad


def _chart(packed: torch.Tensor) -> torch.Tensor:
    """Tangent coordinates xi with exp(xi^) equal to a packed pose (SE(3) logarithm)."""
    rotation = packed[:9].reshape(3, 3)
    translation = packed[9:]
    cos_theta = ((rotation.trace() - 1.0) / 2.0).clamp(-1.0, 1.0)
    theta = torch.arccos(cos_theta)
    skew = (rotation - rotation.T) / 2.0
    if float(theta) < 1e-8:
        omega = torch.stack([skew[2, 1], skew[0, 2], skew[1, 0]])
        return torch.cat([translation, omega])
    omega = theta / torch.sin(theta) * torch.stack([skew[2, 1], skew[0, 2], skew[1, 0]])
    k = torch.tensor([[0.0, -omega[2], omega[1]], [omega[2], 0.0, -omega[0]], [-omega[1], omega[0], 0.0]],
                     dtype=torch.float64, device=packed.device)
    b = (1.0 - torch.cos(theta)) / theta**2
    c = (theta - torch.sin(theta)) / theta**3
    left = torch.eye(3, dtype=torch.float64, device=packed.device) + b * k + c * (k @ k)
    rho = torch.linalg.solve(left, translation)
    return torch.cat([rho, omega])
