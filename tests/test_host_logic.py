"""Host logic without a GPU: contracts, plans, operator schemas and fake kernels,
status decoding, Projector argument handling."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from dpt_b200 import _native as N
from dpt_b200.contracts import ContractError, NumericalError, TrialDomainError, raise_device_status
from dpt_b200.geometry import ConeBeamIntrinsics, RayBundleGeometry, RigidTransform
from dpt_b200.plan import panel_record, plan_rays
from dpt_b200.projection import ProjectionSpec
from dpt_b200.torch import Projector
from dpt_b200.torch import _projection_ops as ops
from dpt_b200.volumes import GridSpec
from scenes import cone_scene, mixed_panels, projector_fixture


def test_status_bits_map_to_reference_error_types():
    raise_device_status(0, "projection")
    with pytest.raises(ContractError, match="invalid rigid pose"):
        raise_device_status(1 | 2, "projection")
    with pytest.raises(TrialDomainError, match="finite and non-negative"):
        raise_device_status(8 | 2, "projection")
    with pytest.raises(NumericalError, match="non-finite"):
        raise_device_status(2, "projection")
    with pytest.raises(NumericalError, match="unknown"):
        raise_device_status(64, "projection")
    assert issubclass(TrialDomainError, NumericalError)


def test_spec_contracts():
    ProjectionSpec(8, sampling_precision="compensated", storage_precision="bfloat16")
    with pytest.raises(ContractError):
        ProjectionSpec(0)
    # reference ProjectionSpec rules (python/dpt/projection.py:113-140)
    with pytest.raises(ContractError, match="FP32 field storage"):
        ProjectionSpec(8, sampling_precision="float32", storage_precision="float16")
    with pytest.raises(ContractError, match="fixed pose"):
        ProjectionSpec(8, sampling_precision="mixed_float32")
    with pytest.raises(ContractError, match="fixed pose"):
        ProjectionSpec(8, sampling_precision="fast_float32", active_pose=False, integration="cell_gauss")
    with pytest.raises(ContractError):
        ProjectionSpec(8, integration="gauss")
    with pytest.raises(ContractError):
        ProjectionSpec(8, field_domain="negative")
    with pytest.raises(ContractError):
        ProjectionSpec(8, validate="sometimes")
    assert ProjectionSpec(8, integration="cell_gauss").arith == N.ARITH_CELLS
    assert ProjectionSpec(8, sampling_precision="fast_float32", active_pose=False).arith == N.ARITH_FAST
    assert ProjectionSpec(8, sampling_precision="float64", storage_precision="bfloat16").field_code == N.BF16
    assert ProjectionSpec(8, field_domain="signed_linear").domain_code == N.DOMAIN_SIGNED
    with pytest.raises(ContractError):
        ProjectionSpec(8, layout="direct", sampling_precision="compensated", storage_precision="float16")
    assert ProjectionSpec(8, sampling_precision="float64").batch_views == 2
    assert ProjectionSpec(8, sampling_precision="float32").batch_views == 8
    assert ProjectionSpec(8, widen_views=30).batch_views == 30


def test_plan_tables():
    grid, geometry, _ = cone_scene()
    plan = plan_rays(grid, geometry)
    assert plan.view_table.shape == (len(geometry.views), N.VIEW_WORDS)
    first = geometry.views[0]
    record = plan.view_table[0]
    np.testing.assert_array_equal(record[0:3], first.source_mm)
    np.testing.assert_array_equal(record[6:9], [x * first.spacing_mm[0] for x in first.u])
    m = np.asarray(plan.object_to_grid).reshape(3, 3)
    p = grid.grid_to_object((2.0, 3.0, 4.0))
    np.testing.assert_allclose(m @ (np.asarray(p) - np.asarray(plan.grid_origin)), (2.0, 3.0, 4.0), atol=1e-12)
    mixed = plan_rays(grid, mixed_panels(grid))
    assert [int(w) for w in mixed.view_table[:, N.VIEW_MODE_WORD]] == [N.PANEL_CONE, N.PANEL_PARALLEL,
                                                                         N.PANEL_CURVED]
    assert mixed.view_table[2, 14] == pytest.approx(80.0)
    bundle = plan_rays(grid, RayBundleGeometry(((0.0, -40.0, 0.0),), ((0.0, 40.0, 1.0),)))
    assert bundle.ray_kind == N.RAYS_BUNDLE and bundle.image_shape == (1,)
    p = plan.problem(17, N.ARITH_F32)
    assert (p.nx, p.ny, p.nz, p.views, p.samples) == (grid.shape[2], grid.shape[1], grid.shape[0],
                                                       len(geometry.views), 17)
    assert len(panel_record(first)) == N.VIEW_WORDS


def test_configuration_round_trip_and_workspace_key():
    grid, geometry, _, samples = projector_fixture()
    value = ops.configuration(grid, geometry, samples, "float32")
    decoded_grid, decoded_geometry, decoded_samples, precision = ops.decode(value)
    assert decoded_grid == grid and decoded_geometry == geometry
    assert decoded_samples == samples and precision == "float32"
    with pytest.raises(ContractError):
        ops.configuration(grid, geometry, samples, "float16")


def test_fake_kernels_on_meta_tensors():
    grid, geometry, _, samples = projector_fixture()
    value = ops.configuration(grid, geometry, samples, "float64")
    field = torch.empty(grid.shape, dtype=torch.float32, device="meta")
    poses = torch.empty((len(geometry.views), 12), dtype=torch.float64, device="meta")
    image = torch.ops.dpt.project(field, poses, value, True, True)
    assert image.shape == geometry.shape and image.dtype == torch.float64 and image.device.type == "meta"
    cot = torch.empty(geometry.shape, dtype=torch.float64, device="meta")
    grad, pose_grad = torch.ops.dpt.project_vjp(field, poses, cot, value, True, False)
    assert grad.shape == field.shape and pose_grad.shape == (0,)
    out = torch.empty(geometry.shape, dtype=torch.float64, device="meta")
    torch.ops.dpt.project_out(field, poses, value, out)
    with pytest.raises(ContractError, match="poses"):
        torch.ops.dpt.project(field, poses[:1], value, False, False)
    with pytest.raises(ContractError, match="cotangent"):
        torch.ops.dpt.project_vjp(field, poses, cot.float(), value, True, False)


def test_projector_arguments_and_cpu_rejection():
    grid, geometry, field, samples = projector_fixture()
    module = Projector(grid=grid, geometry=geometry, precision="fp32", samples_per_ray=samples)
    assert isinstance(module, torch.nn.Module) and module.samples_per_ray == samples
    assert Projector(grid=grid, geometry=geometry).samples_per_ray == 1024
    stepped = Projector(grid=grid, geometry=geometry, step_mm=0.2)
    nz, ny, nx = grid.shape
    expected = math.ceil(math.hypot(nx * grid.spacing_mm[0], ny * grid.spacing_mm[1], nz * grid.spacing_mm[2]) / 0.2)
    assert stepped.samples_per_ray == expected
    with pytest.raises(ContractError, match="choose samples_per_ray or step_mm"):
        Projector(grid=grid, geometry=geometry, samples_per_ray=4, step_mm=0.2)
    with pytest.raises(ContractError, match="precision"):
        Projector(grid=grid, geometry=geometry, precision="fp16")
    anchor = torch.nn.Parameter(torch.tensor(RigidTransform().packed(), dtype=torch.float64))
    with_anchor = Projector(grid=grid, geometry=geometry, anchor=anchor)
    assert dict(with_anchor.named_parameters())["anchor"] is anchor
    cpu_field = torch.tensor(field["field"])
    with pytest.raises(ContractError, match="CUDA"):
        module(cpu_field)
    with pytest.raises(ContractError, match="grid shape"):
        module(cpu_field[:1])
    with pytest.raises(ContractError, match="float32"):
        module(cpu_field.double())


def test_cone_batch_helpers():
    intrinsics = ConeBeamIntrinsics(1000.0, 1500.0, (512, 512), (0.8, 0.8))
    batch = intrinsics.batch(tuple(2 * math.pi * k / 360 for k in range(360)))
    assert batch.shape == (360, 512, 512)
    grid = GridSpec((4, 4, 4), (1.0, 1.0, 1.0))
    plan = plan_rays(grid, batch)
    assert plan.rays == 360 * 512 * 512


def test_packed_forward_rejects_empty_oversized_and_foreign_calls_before_any_launch():
    from dpt_b200.projection import forward_packed

    with pytest.raises(ContractError):
        forward_packed([])
    with pytest.raises(ContractError):
        forward_packed([(None, None, None)] * (N.MAX_PACK + 1))
    with pytest.raises(ContractError):  # not a projection workspace
        forward_packed([("workspace", torch.zeros(2), torch.zeros(12, dtype=torch.float64))])
