"""The pose VJP that allocates nothing (dpt_b200_pose_vjp_fixed) against the allocating path.

That entry point serves callers that cannot call cudaMalloc while they run: tracking or
guidance loops that reserve their device memory at start-up and hosts that own all GPU
memory.  Its per-block partials live in a fixed device array inside the library, so two
calls in a row must both reproduce the pose gradient of dpt_b200_vjp + dpt_b200_finish_pose
(with caller scratch, the same direct-gather sampling); this file is collected last so a
failure here comes after every other test has run.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from dpt_b200 import _native as N
from dpt_b200.plan import plan_rays
from dpt_b200.projection import ProjectionSpec, ProjectionWorkspace
from scenes import cone_scene, poses_for

pytestmark = pytest.mark.gpu

CASES = [
    ("float32", "midpoint", 12),
    ("float32", "midpoint", 6),
    ("float64", "midpoint", 12),
    ("compensated", "midpoint", 12),
    ("float64", "cell_gauss", 6),
]


@pytest.mark.parametrize("sampling, integration, components", CASES)
def test_fixed_scratch_pose_vjp_matches_the_allocating_entry_point(sampling, integration, components):
    grid, geometry, values = cone_scene(views=3, detector=(40, 36))
    poses = torch.tensor(poses_for(3, seed=12), dtype=torch.float64, device="cuda:0")
    precision = "float64" if sampling == "float64" else "float32"
    # the allocating path with the same direct gathers the fixed entry point uses
    spec = ProjectionSpec(57, precision=precision, sampling_precision=sampling, integration=integration,
                          layout="direct")
    workspace = ProjectionWorkspace(plan_rays(grid, geometry), spec, "cuda:0")
    field = torch.tensor(values, device="cuda:0")
    dtype = torch.float64 if precision == "float64" else torch.float32
    cotangent = torch.linspace(-0.7, 1.1, workspace.plan.rays, dtype=dtype, device="cuda:0")
    cotangent = cotangent.reshape(workspace.plan.image_shape)
    _, expected = workspace.vjp(field, poses, cotangent, volume=False,
                                pose="matrix" if components == 12 else "tangent")

    lib = N.library()
    status = torch.zeros(3, dtype=torch.int32, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # the fixed array keeps the previous call's contents
        out = torch.full((3, components), float("nan"), dtype=torch.float64, device="cuda:0")
        code = lib.dpt_b200_pose_vjp_fixed(workspace.problem, workspace.rays(poses), field.data_ptr(),
                                           cotangent.data_ptr(), components, out.data_ptr(),
                                           status.data_ptr(), stream)
        assert code == 0, lib.dpt_b200_error_string(code)
        torch.cuda.synchronize()
        assert status.cpu().tolist() == [0, 0, 0]
        np.testing.assert_allclose(out.cpu().numpy(), expected.cpu().numpy(), rtol=1e-12, atol=1e-15)


def test_fixed_scratch_rejects_work_beyond_its_capacity():
    """A 4096 x 4096 single view needs 65536 blocks x 12 partials, more than the array holds:
    the call returns DPT_E_CAPACITY before any launch.  Every pointer is a real device buffer
    of the size the call would use, so a regression returns a wrong code or writes values
    here, never an out-of-range address."""
    grid, geometry, values = cone_scene(views=1, detector=(40, 36))
    workspace = ProjectionWorkspace(plan_rays(grid, geometry), ProjectionSpec(9, sampling_precision="float32"),
                                    "cuda:0")
    big = N.Problem.from_buffer_copy(workspace.problem)
    big.rows = big.cols = 4096
    device = "cuda:0"
    field = torch.tensor(values, device=device)
    cotangent = torch.zeros(4096 * 4096, dtype=torch.float32, device=device)
    poses = torch.tensor(poses_for(1, seed=3), dtype=torch.float64, device=device)
    out = torch.full((1, 12), float("nan"), dtype=torch.float64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    rays = workspace.rays(poses)
    code = N.library().dpt_b200_pose_vjp_fixed(big, rays, field.data_ptr(), cotangent.data_ptr(), 12,
                                               out.data_ptr(), status.data_ptr(),
                                               torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert code == -7 and N.library().dpt_b200_error_string(code) == b"a fixed-capacity buffer is too small"
    assert int(status.item()) == 0
    assert bool(torch.isnan(out).all())
