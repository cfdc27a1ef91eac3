"""Projector / dpt::* operators on the GPU against the reference's independent matrix,
finite differences and its behavioural tests (tests/python/warp_cpu/test_projector_workflow.py,
tests/python/warp_cpu/test_torch_projection_registration.py)."""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest
import torch

from dpt_b200.api import project
from dpt_b200.contracts import ContractError, NumericalError, TrialDomainError
from dpt_b200.geometry import RigidTransform
from dpt_b200.imaging import ImagingMetadata, ImagingVolume
from dpt_b200.torch import Projector, compose_pose
from scenes import cone_scene, projector_fixture

pytestmark = pytest.mark.gpu
DEVICE = "cuda:0"


def problem():
    grid, geometry, data, samples = projector_fixture()
    field = torch.tensor(data["field"], device=DEVICE)
    operator = torch.tensor(data["matrix_47"], dtype=torch.float64, device=DEVICE)
    return grid, geometry, field, samples, operator


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_images_and_volume_gradient_match_independent_matrix(precision):
    grid, geometry, field, samples, operator = problem()
    module = Projector(grid=grid, geometry=geometry, precision=precision, samples_per_ray=samples)
    field.requires_grad_()
    image = module(field)
    assert tuple(image.shape) == geometry.shape
    assert image.dtype == (torch.float32 if precision == "fp32" else torch.float64)
    expected = operator @ field.detach().reshape(-1).double()
    tolerance = 5e-6 if precision == "fp32" else 2e-11
    torch.testing.assert_close(image.reshape(-1).double(), expected, rtol=tolerance, atol=tolerance)
    seed = torch.linspace(-0.5, 0.8, image.numel(), dtype=image.dtype, device=DEVICE).reshape(image.shape)
    image.backward(seed)
    torch.testing.assert_close(field.grad.reshape(-1).double(), operator.T @ seed.reshape(-1).double(),
                               rtol=5e-6, atol=5e-7)


def test_pose_tangent_gradcheck_and_packed_pose_equivalence():
    grid, geometry, field, samples, _ = problem()
    module = Projector(grid=grid, geometry=geometry, precision="fp64", samples_per_ray=samples)
    tangent = torch.tensor([0.03, -0.02, 0.01, 0.04, -0.03, 0.02], dtype=torch.float64, device=DEVICE,
                           requires_grad=True)
    assert torch.autograd.gradcheck(lambda value: module(field, value), (tangent,), eps=2e-5, atol=2e-6,
                                    rtol=2e-5)
    identity = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=DEVICE)
    torch.testing.assert_close(module(field, tangent), module(field, packed_pose=compose_pose(identity, tangent)))
    with pytest.raises(ContractError, match="choose pose or packed_pose"):
        module(field, tangent, packed_pose=identity)


def test_fp32_pose_gradient_agrees_with_fp64():
    grid, geometry, field, samples, _ = problem()
    tangent = torch.tensor([0.03, -0.02, 0.01, 0.04, -0.03, 0.02], dtype=torch.float64, device=DEVICE,
                           requires_grad=True)
    gradients = []
    for precision in ("fp32", "fp64"):
        module = Projector(grid=grid, geometry=geometry, precision=precision, samples_per_ray=samples)
        image = module(field, tangent)
        seed = torch.linspace(-0.5, 0.8, image.numel(), device=DEVICE).reshape(image.shape)
        gradients.append(torch.autograd.grad((image * seed).sum(), tangent)[0])
    torch.testing.assert_close(gradients[0], gradients[1], rtol=2e-4, atol=5e-6)


@pytest.mark.parametrize("mutation", ["field", "packed_pose"])
def test_input_mutation_before_backward_is_detected(mutation):
    grid, geometry, field, samples, _ = problem()
    module = Projector(grid=grid, geometry=geometry, precision="fp64", samples_per_ray=samples)
    field.requires_grad_()
    pose = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=DEVICE)
    image = module(field, packed_pose=pose)
    with torch.no_grad():
        if mutation == "field":
            field.add_(0.01)
        else:
            pose[9].add_(0.01)
    with pytest.raises(RuntimeError, match="modified by an inplace operation"):
        image.sum().backward()


def test_repeated_calls_keep_outputs_separate():
    grid, geometry, field, samples, operator = problem()
    module = Projector(grid=grid, geometry=geometry, precision="fp64", samples_per_ray=samples)
    field.requires_grad_()
    first = module(field)
    saved = first.detach().clone()
    second = module(0.5 * field)
    assert first.data_ptr() != second.data_ptr()
    torch.testing.assert_close(first, saved)
    torch.testing.assert_close(second, 0.5 * first)
    (first.sum() + second.sum()).backward()
    torch.testing.assert_close(field.grad.reshape(-1).double(), 1.5 * operator.sum(0), rtol=4e-6, atol=1e-7)


def test_inference_out_buffer():
    grid, geometry, field, samples, _ = problem()
    module = Projector(grid=grid, geometry=geometry, precision="fp64", samples_per_ray=samples)
    expected = module(field)
    out = torch.full_like(expected, -123.0)
    assert module(field, out=out) is out
    torch.testing.assert_close(out, expected)
    field.requires_grad_()
    out.fill_(-123.0)
    with pytest.raises(ContractError, match="inference buffer"):
        module(field, out=out)
    torch.testing.assert_close(out, torch.full_like(out, -123.0))
    with torch.no_grad():
        assert module(field, out=out) is out
    torch.testing.assert_close(out, expected)


def test_functional_project_and_prepared_tensor():
    grid, geometry, field, samples, _ = problem()
    volume = ImagingVolume(field.cpu().numpy(), grid, ImagingMetadata("synthetic", "RAS", "mm^-1"))
    module = Projector(grid=grid, geometry=geometry, precision="fp64", samples_per_ray=samples)
    resident = field.clone().requires_grad_()
    expected = module(resident)
    torch.testing.assert_close(project(volume, geometry, device=DEVICE, precision="fp64", samples_per_ray=samples),
                               expected)
    again = project(resident, prepared=module)
    torch.testing.assert_close(again, expected)
    again.sum().backward()
    assert resident.grad is not None
    with pytest.raises(ContractError, match="precision"):
        project(resident, prepared=module, precision="fp32")
    with pytest.raises(ContractError, match="convert HU"):
        project(replace(volume, metadata=replace(volume.metadata, value_units="HU")), geometry)


def test_invalid_inputs_raise_typed_errors_and_the_next_call_recovers():
    grid, geometry, field, samples, _ = problem()
    module = Projector(grid=grid, geometry=geometry, precision="fp32", samples_per_ray=samples)
    good = module(field)
    poisoned = field.clone()
    poisoned.view(-1)[3] = float("inf")
    with pytest.raises(TrialDomainError):
        module(poisoned)
    negative = field.clone()
    negative.view(-1)[0] = -1e-3
    with pytest.raises(TrialDomainError, match="non-negative"):
        module(negative)
    skewed = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=DEVICE)
    skewed[1] = 1e-3
    with pytest.raises(ContractError, match="rigid pose"):
        module(field, packed_pose=skewed)
    torch.testing.assert_close(module(field), good)
    field.requires_grad_()
    image = module(field)
    cot = torch.ones_like(image)
    cot.view(-1)[5] = float("nan")
    with pytest.raises(NumericalError):
        image.backward(cot)
    image = module(field)
    image.backward(torch.ones_like(image))
    assert torch.isfinite(field.grad).all()


def test_half_storage_fields_through_the_projector():
    """FP16/BF16 fields run the compensated arithmetic on their decoded values: bit-identical
    to the compensated form on the decoded FP32 field, and within 1e-5 relative L2 of the
    FP32 reference-arithmetic projector."""
    from dpt_b200.plan import plan_rays
    from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace

    grid, geometry, values = cone_scene()
    module = Projector(grid=grid, geometry=geometry, precision="fp32", samples_per_ray=64)
    compensated = ProjectionWorkspace(plan_rays(grid, geometry),
                                      ProjectionSpec(64, sampling_precision="compensated"), DEVICE)
    identity = torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=DEVICE)
    poses = identity.expand(len(geometry.views), 12).contiguous()
    reference_field = torch.tensor(values, device=DEVICE)
    for dtype in (torch.bfloat16, torch.float16):
        half = reference_field.to(dtype).requires_grad_()
        decoded = half.detach().float().requires_grad_()
        image = module(half)
        torch.testing.assert_close(image, compensated.forward(decoded.detach(), poses), rtol=0, atol=0)
        baseline = module(decoded)
        error = (image - baseline).norm() / baseline.norm()
        assert error < 1e-5, float(error)
        image.sum().backward()
        baseline.sum().backward()
        assert half.grad.dtype == dtype
        torch.testing.assert_close(half.grad.float(), decoded.grad, rtol=1e-2, atol=1e-3)


def test_step_mm_and_registered_anchor_parameter():
    import math

    grid, geometry, field, _, _ = problem()
    anchor = torch.nn.Parameter(torch.tensor(RigidTransform().packed(), dtype=torch.float64, device=DEVICE))
    module = Projector(grid=grid, geometry=geometry, precision="fp64", step_mm=0.2, anchor=anchor)
    nz, ny, nx = grid.shape
    samples = math.ceil(math.hypot(nx * grid.spacing_mm[0], ny * grid.spacing_mm[1], nz * grid.spacing_mm[2]) / 0.2)
    explicit = Projector(grid=grid, geometry=geometry, precision="fp64", samples_per_ray=samples)
    assert module.samples_per_ray == samples
    torch.testing.assert_close(module(field), explicit(field))
    module(field).sum().backward()
    assert anchor.grad is not None and torch.isfinite(anchor.grad).all()
    np.testing.assert_array_equal(anchor.grad.shape, (12,))
