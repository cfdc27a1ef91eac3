"""The compensated precision form (no reference counterpart) checked against the reference's
strict FP64 arithmetic on the CPU oracle: the cell-run closed form must stay within the
form's precision bar on cone scans and on adversarial bundles (axis-parallel rays, rays
through cell planes, single-voxel and flat grids, 1 to 513 samples), and its volume VJP must
be the adjoint of its forward.  Oracle-only: no GPU.
"""

from __future__ import annotations

import numpy as np
import pytest

from dpt_b200.geometry import RayBundleGeometry
from dpt_b200.plan import plan_rays
from dpt_b200.volumes import GridSpec
from oracle import oracle as O
from scenes import cone_scene, poses_for

IDENTITY = np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0])


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("samples", [7, 53, 1024])
def test_cone_scan_against_strict_fp64(samples):
    grid, geometry, values = cone_scene()
    plan = plan_rays(grid, geometry)
    poses = poses_for(len(geometry.views), seed=2)
    strict, _ = O.forward(plan, values, poses, samples=samples, arith=O.ARITH_F64, image_dtype=O.F64)
    image, status = O.forward(plan, values, poses, samples=samples, arith=O.ARITH_F32C)
    assert not status.any()
    assert rel_l2(image, strict) < 1e-6
    seed = np.random.default_rng(1).uniform(-1, 1, plan.rays).astype(np.float32)
    flags = O.VJP_VOLUME | O.VJP_POSE6
    volume, pose, status = O.vjp(plan, values, poses, seed, samples=samples, flags=flags,
                                 arith=O.ARITH_F32C)
    assert not status.any()
    volume64, pose64, _ = O.vjp(plan, values, poses, seed.astype(np.float64), samples=samples,
                                flags=flags, arith=O.ARITH_F64, image_dtype=O.F64)
    assert rel_l2(volume, volume64) < 1e-5
    assert rel_l2(pose, pose64) < 1e-5
    # adjoint identity <A v, s> = <v, A^T s> of the form's own forward and volume VJP
    left = float(image.astype(np.float64) @ seed.astype(np.float64))
    right = float(values.reshape(-1).astype(np.float64) @ volume)
    assert abs(left - right) <= 1e-6 * abs(left)


def _adversarial_bundle(shape, rng):
    nz, ny, nx = shape
    extent = np.array([nx * 1.0, ny * 0.7, nz * 1.3])
    sources, ends = [], []
    for k in range(120):
        start = rng.uniform(-1, 1, 3) * extent
        kind = k % 3
        if kind == 0:  # parallel to one axis
            axis = rng.integers(3)
            end = start.copy()
            start[axis], end[axis] = -3 * extent[axis], 3 * extent[axis]
        elif kind == 1:  # through integer planes
            start = np.round(start)
            end = start + 4 * (np.round(rng.uniform(-1, 1, 3)) - 2 * start)
        else:
            start, end = 3 * start, rng.uniform(-1, 1, 3) * extent * 3
        if np.linalg.norm(end - start) < 1e-6:
            end = start + np.array([1.0, 0.5, 0.25])
        sources.append(tuple(start))
        ends.append(tuple(end))
    return RayBundleGeometry(tuple(sources), tuple(ends))


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 3, 5), (4, 1, 6), (5, 6, 7)])
def test_adversarial_rays_against_strict_fp64(shape):
    rng = np.random.default_rng(sum(shape))
    grid = GridSpec(shape, (1.0, 0.7, 1.3))
    plan = plan_rays(grid, _adversarial_bundle(shape, rng))
    values = rng.uniform(0, 1, shape).astype(np.float32)
    for samples in (1, 3, 64, 513):
        strict, _ = O.forward(plan, values, IDENTITY, samples=samples, arith=O.ARITH_F64,
                              image_dtype=O.F64)
        image, status = O.forward(plan, values, IDENTITY, samples=samples, arith=O.ARITH_F32C)
        assert not status.any()
        assert np.abs(image - strict).max() <= 1e-6 * np.abs(strict).max()
        seed = rng.uniform(-1, 1, plan.rays).astype(np.float32)
        volume, _, _ = O.vjp(plan, values, IDENTITY, seed, samples=samples, flags=O.VJP_VOLUME,
                             arith=O.ARITH_F32C)
        volume64, _, _ = O.vjp(plan, values, IDENTITY, seed.astype(np.float64), samples=samples,
                               flags=O.VJP_VOLUME, arith=O.ARITH_F64, image_dtype=O.F64)
        assert np.abs(volume - volume64).max() <= 1e-6 * np.abs(volume64).max()
