"""The packed forward (``dpt_b200_forward_packed``): one launch over the
(view, tile) blocks of several workspaces of one sampling arithmetic, field layout and image
dtype.  Every image equals that workspace's own ``forward`` bit for bit (the same per-ray
code and order of summation) and the oracle's image on the same inputs; mixed scenes (cone,
parallel and curved panels, different grids, sample counts and view counts) go in one pack.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from dpt_b200 import _native as N
from dpt_b200.contracts import ContractError
from dpt_b200.plan import plan_rays
from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace, forward_packed
from oracle import oracle as O
from scenes import cone_scene, mixed_panels, poses_for, rotated_grid

pytestmark = pytest.mark.gpu
DEVICE = "cuda:0"

ARITH = {"float32": O.ARITH_F32, "float64": O.ARITH_F64, "compensated": O.ARITH_F32C}


def scenes():
    """Five differently shaped problems: cone scenes of several grids, views and detectors,
    and the mixed cone / parallel / curved panel set."""
    out = [cone_scene(),
           cone_scene(shape=(9, 12, 10), spacing=(0.9, 1.4, 1.0), views=3, detector=(13, 17)),
           cone_scene(shape=(20, 8, 11), views=7, detector=(32, 8)),
           cone_scene(shape=(6, 6, 6), views=1, detector=(5, 70))]
    grid = rotated_grid((10, 11, 12), (1.1, 0.9, 1.3))
    rng = np.random.default_rng(5)
    out.append((grid, mixed_panels(grid), rng.uniform(0.0, 0.02, size=grid.shape).astype(np.float32)))
    return out


def make(grid, geometry, samples, sampling, storage="float32", layout="replicated"):
    precision = "float64" if sampling == "float64" else "float32"
    spec = ProjectionSpec(samples, precision=precision, sampling_precision=sampling,
                          storage_precision=storage, layout=layout)
    return ProjectionWorkspace(plan_rays(grid, geometry), spec, DEVICE)


@pytest.mark.parametrize("sampling,storage,layout", [
    ("float32", "float32", "replicated"), ("float32", "float32", "direct"),
    ("compensated", "bfloat16", "replicated"), ("float64", "float32", "replicated")])
def test_packed_images_equal_each_workspace_forward_and_the_oracle(sampling, storage, layout):
    calls, expected = [], []
    for k, (grid, geometry, values) in enumerate(scenes()):
        samples = (23, 61, 128, 7, 40)[k]
        ws = make(grid, geometry, samples, sampling, storage, layout)
        poses = poses_for(ws.plan.views, seed=k + 2)
        dtype = torch.bfloat16 if storage == "bfloat16" else torch.float32
        field = torch.tensor(values, device=DEVICE).to(dtype)
        pose = torch.tensor(poses, dtype=torch.float64, device=DEVICE)
        calls.append((ws, field, pose))
        expected.append(ws.forward(field, pose).clone())
    images = forward_packed(calls)
    torch.cuda.synchronize()
    for (ws, field, pose), got, own in zip(calls, images, expected):
        assert torch.equal(got, own)
        stored = field.float().cpu().numpy()
        oracle_image, status = O.forward(ws.plan, stored, pose.cpu().numpy(), samples=ws.spec.samples_per_ray,
                                         arith=ARITH[sampling],
                                         image_dtype=O.F64 if sampling == "float64" else O.F32)
        assert not status.any()
        np.testing.assert_array_equal(got.cpu().numpy().reshape(-1), oracle_image)


def test_packed_forward_fills_given_outputs_and_repeats_a_workspace():
    grid, geometry, values = cone_scene()
    ws = make(grid, geometry, 33, "float32")
    field = torch.tensor(values, device=DEVICE)
    poses = [torch.tensor(poses_for(len(geometry.views), seed=s), dtype=torch.float64, device=DEVICE)
             for s in (1, 2, 3)]
    own = [ws.forward(field, p).clone() for p in poses]
    outs = [torch.full_like(own[0], float("nan")) for _ in poses]
    got = forward_packed([(ws, field, p, o) for p, o in zip(poses, outs)])
    torch.cuda.synchronize()
    for g, o, e in zip(got, outs, own):
        assert g.data_ptr() == o.data_ptr()
        assert torch.equal(o, e)


def test_packed_forward_of_the_largest_pack():
    grid, geometry, values = cone_scene(views=2, detector=(9, 10))
    ws = make(grid, geometry, 19, "float32")
    field = torch.tensor(values, device=DEVICE)
    poses = [torch.tensor(poses_for(2, seed=s), dtype=torch.float64, device=DEVICE) for s in range(N.MAX_PACK)]
    own = [ws.forward(field, p).clone() for p in poses]
    got = forward_packed([(ws, field, p) for p in poses])
    torch.cuda.synchronize()
    assert all(torch.equal(g, e) for g, e in zip(got, own))


def test_packed_forward_rejects_mixed_classes_and_pack_sizes():
    grid, geometry, values = cone_scene()
    field = torch.tensor(values, device=DEVICE)
    pose = torch.tensor(poses_for(len(geometry.views)), dtype=torch.float64, device=DEVICE)
    a = make(grid, geometry, 17, "float32")
    b = make(grid, geometry, 17, "float64")
    with pytest.raises(ContractError):
        forward_packed([(a, field, pose), (b, field, pose)])
    with pytest.raises(ContractError):
        forward_packed([])
    with pytest.raises(ContractError):  # one sampling copy per workspace
        forward_packed([(a, field, pose), (a, field * 2, pose)])
    with pytest.raises(ContractError):
        forward_packed([(a, field, pose)] * (N.MAX_PACK + 1))
