"""Geometry objects and the SE(3) chart against the reference's own outputs (fixtures)."""

from __future__ import annotations

import json
import math

import numpy as np
import pytest
import torch

from dpt_b200.contracts import ContractError
from dpt_b200.geometry import (
    BatchedGeometry,
    ConeBeamIntrinsics,
    CurvedDetectorGeometry,
    DetectorGeometry,
    ParallelGeometry,
    RayBundleGeometry,
    RigidTransform,
    chart_gradient,
    compose_pose,
    right_jacobian_se3,
)
from dpt_b200.imaging import ImagingMetadata, ImagingVolume, ct_to_attenuation, standard_views
from dpt_b200.torch.geometry import compose_pose as torch_compose
from dpt_b200.volumes import GridSpec
from scenes import GOLDEN, grid_from

FACTS = json.loads((GOLDEN / "facts.json").read_text())


@pytest.mark.parametrize("index", range(4))
def test_se3_chart_matches_reference(index):
    anchor = RigidTransform(tuple(FACTS["chart"]["anchor"][:9]), tuple(FACTS["chart"]["anchor"][9:]))
    case = FACTS["chart"]["cases"][index]
    xi = tuple(case["increment"])
    np.testing.assert_allclose(compose_pose(anchor, xi).packed(), case["composed"], rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(right_jacobian_se3(xi), case["jacobian"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(chart_gradient(xi, tuple(case["right_gradient"])), case["chart_gradient"],
                               rtol=1e-12, atol=1e-13)
    # the Torch chart (matrix exponential) agrees with the closed form
    packed = torch_compose(torch.tensor(FACTS["chart"]["anchor"], dtype=torch.float64),
                           torch.tensor(xi, dtype=torch.float64))
    np.testing.assert_allclose(packed.numpy(), case["composed"], rtol=1e-10, atol=1e-11)


def test_torch_chart_gradient_is_the_right_jacobian_transpose():
    xi = torch.tensor([0.3, -0.2, 0.1, 0.4, -0.7, 0.2], dtype=torch.float64, requires_grad=True)
    anchor = torch.tensor(RigidTransform().packed(), dtype=torch.float64)
    packed = torch_compose(anchor, xi)
    # local-right perturbation delta: G(xi) exp(delta^); first order d packed = ...
    g_right = torch.tensor([0.5, -1.0, 0.25, 0.3, 0.2, -0.4], dtype=torch.float64)
    # packed cotangent whose local-right pullback is g_right: translation rows R g_t,
    # rotation rows from R [w]x with w = g_r / 2 contracted over both off-diagonals
    rotation = packed.detach()[:9].reshape(3, 3)
    cot = torch.zeros(12, dtype=torch.float64)
    cot[9:] = rotation @ g_right[:3]

    def skew(w):
        return torch.tensor([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]], dtype=torch.float64)

    cot[:9] = (rotation @ skew(g_right[3:]) / 2.0).reshape(-1)
    (packed * cot).sum().backward()
    expected = chart_gradient(tuple(xi.detach().tolist()), tuple(g_right.tolist()))
    np.testing.assert_allclose(xi.grad.numpy(), expected, rtol=1e-10, atol=1e-12)


def test_cone_views_and_projection_matrix_match_reference():
    intrinsics = ConeBeamIntrinsics(500.0, 1000.0, (64, 64), (1.5, 1.5), (0.7, -0.4), (1.0, 2.0, 3.0))
    for record in FACTS["cone"]["views"]:
        panel = intrinsics.view(record["angle"])
        np.testing.assert_allclose(panel.source_mm, record["source_mm"], rtol=1e-14, atol=1e-12)
        np.testing.assert_allclose(panel.origin_mm, record["origin_mm"], rtol=1e-14, atol=1e-12)
        np.testing.assert_allclose(panel.u, record["u"], atol=1e-15)
        np.testing.assert_allclose(panel.v, record["v"], atol=1e-15)
        np.testing.assert_allclose(panel.pixel_centre(3, 5), record["centre_3_5"], rtol=1e-14, atol=1e-12)
        np.testing.assert_allclose(panel.project_point((10.0, -4.0, 7.0)), record["project_point"], rtol=1e-12)
    grid = grid_from(FACTS["cone"]["standard_grid"])
    views = standard_views(grid, shape=(32, 48))
    for panel, record in zip(views.views, FACTS["cone"]["standard_views"], strict=True):
        np.testing.assert_allclose(panel.source_mm, record["source_mm"], rtol=1e-13, atol=1e-10)
        np.testing.assert_allclose(panel.origin_mm, record["origin_mm"], rtol=1e-13, atol=1e-10)
        np.testing.assert_allclose(panel.spacing_mm, record["spacing_mm"], rtol=1e-14)


def test_panel_contracts_and_bundles():
    with pytest.raises(ContractError, match="unit length"):
        DetectorGeometry((0.0, -5.0, 0.0), (0, 5.0, 0), (2.0, 0.0, 0.0), (0.0, 0.0, 1.0), (1.0, 1.0), (2, 2))
    with pytest.raises(ContractError, match="outside the detector plane"):
        DetectorGeometry((0.0, 5.0, 0.0), (0, 5.0, 0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (1.0, 1.0), (2, 2))
    with pytest.raises(ContractError, match="orthonormal"):
        RigidTransform((1.0, 0.1, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0))
    with pytest.raises(ContractError, match="right-handed"):
        RigidTransform((-1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0))
    panel = DetectorGeometry((0.0, -50.0, 0.0), (-2.0, 30.0, -1.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (1.0, 0.5), (3, 5))
    bundle = RayBundleGeometry.from_views((panel, panel))
    assert bundle.pixels == 30 and bundle.view_offsets == (0, 15, 30)
    assert bundle.segment(7) == (panel.source_mm, panel.pixel_centre(1, 2))
    with pytest.raises(ContractError):
        RayBundleGeometry(((0.0, 0.0, 0.0),), ((0.0, 0.0, 0.0),))
    batch = BatchedGeometry((panel, panel))
    assert batch.shape == (2, 3, 5) and batch.pixels == 30
    astra = batch.to_astra_vectors()
    back = BatchedGeometry.from_astra_vectors(astra)
    for a, b in zip(batch.views, back.views, strict=True):
        np.testing.assert_allclose(a.origin_mm, b.origin_mm, atol=1e-12)
        np.testing.assert_allclose(a.spacing_mm, b.spacing_mm, atol=1e-12)
    with pytest.raises(ContractError, match="share"):
        BatchedGeometry((panel, DetectorGeometry((0.0, -50.0, 0.0), (-2.0, 30.0, -1.0), (1.0, 0.0, 0.0),
                                                 (0.0, 0.0, 1.0), (1.0, 0.5), (4, 5))))


def test_parallel_and_curved_panels():
    parallel = ParallelGeometry((0.0, 10.0, 0.0), (0.0, 1.0, 0.0), 40.0, (1.0, 0.0, 0.0), (0.0, 0.0, 1.0),
                                (1.0, 1.0), (2, 3))
    source, end = parallel.segment(1, 2)
    np.testing.assert_allclose(end, (2.0, 10.0, 1.0))
    np.testing.assert_allclose(source, (2.0, -30.0, 1.0))
    curved = CurvedDetectorGeometry((0.0, 0.0, 0.0), (0.0, 100.0, 0.0), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0),
                                    (1.0, 1.0), (1, 3))
    assert curved.radius_mm == pytest.approx(100.0)
    point = curved.pixel_centre(0, 2)
    assert math.dist(point, (0.0, 0.0, 0.0)) == pytest.approx(100.0)
    assert math.atan2(point[0], point[1]) == pytest.approx(0.02)


def test_grid_maps_and_ct_conversion():
    angle = 0.4
    c, s = math.cos(angle), math.sin(angle)
    grid = GridSpec((3, 4, 5), (0.5, 0.7, 1.1), (1.0, -2.0, 3.0), (c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0))
    point = grid.grid_to_object((1.5, 2.0, 0.5))
    np.testing.assert_allclose(grid.object_to_grid(point), (1.5, 2.0, 0.5), atol=1e-12)
    m = np.asarray(grid.object_to_grid_matrix()).reshape(3, 3)
    np.testing.assert_allclose(m @ (np.asarray(point) - grid.origin_mm), (1.5, 2.0, 0.5), atol=1e-12)
    hu = np.asarray([[[-1000.0, 0.0], [1000.0, -1500.0]]])
    volume = ImagingVolume(hu, GridSpec((1, 2, 2), (1.0, 1.0, 1.0)), ImagingMetadata("synthetic", "RAS", "HU"))
    mu = ct_to_attenuation(volume, energy_kev=60.0)
    np.testing.assert_allclose(mu.values.reshape(-1), [0.0, 0.02059, 0.04118, 0.0], rtol=1e-7)
    assert mu.values.dtype == np.float32 and mu.metadata.value_units == "mm^-1"
    with pytest.raises(ContractError):
        ct_to_attenuation(volume, energy_kev=80.0)
