"""Sharded multiview VJP on two gloo ranks (CPU): each rank differentiates its own views
with the oracle, the volume gradients are all-reduced, and the result equals the
single-process gradient over all views; pose gradients stay per view."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dpt_b200.contracts import ContractError
from dpt_b200.distributed import view_range


def test_view_ranges_partition_the_views():
    for views, world in ((360, 1), (360, 2), (360, 8), (7, 3), (5, 5)):
        ranges = [view_range(views, r, world) for r in range(world)]
        assert [i for block in ranges for i in block] == list(range(views))
        assert max(len(b) for b in ranges) - min(len(b) for b in ranges) <= 1
    with pytest.raises(ContractError):
        view_range(2, 0, 3)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, results) -> None:
    import torch
    import torch.distributed as dist

    from dpt_b200.distributed import reduce_volume_gradient
    from dpt_b200.geometry import BatchedGeometry
    from dpt_b200.plan import plan_rays
    from oracle import oracle as O
    from scenes import cone_scene, poses_for

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grid, geometry, values = cone_scene(views=5)
        poses = poses_for(5, seed=8)
        seed = np.random.default_rng(4).uniform(-1, 1, (5, 20, 24)).astype(np.float32)
        block = view_range(5, rank, world)
        local = BatchedGeometry(tuple(geometry.views[v] for v in block))
        plan = plan_rays(grid, local)
        volume, pose, _ = O.vjp(plan, values, poses[block.start:block.stop], seed[block.start:block.stop],
                                samples=33, flags=O.VJP_VOLUME | O.VJP_POSE6, threads=1)
        gradient = torch.from_numpy(volume)
        reduce_volume_gradient(gradient)
        poses_all = [None] * world
        dist.all_gather_object(poses_all, (block.start, pose))
        if rank == 0:
            results.put((gradient.numpy().copy(), poses_all))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_vjp_equals_single_process():
    from dpt_b200.plan import plan_rays
    from oracle import oracle as O
    from scenes import cone_scene, poses_for

    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    gradient, poses_all = results.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    grid, geometry, values = cone_scene(views=5)
    poses = poses_for(5, seed=8)
    seed = np.random.default_rng(4).uniform(-1, 1, (5, 20, 24)).astype(np.float32)
    volume, pose, _ = O.vjp(plan_rays(grid, geometry), values, poses, seed, samples=33,
                            flags=O.VJP_VOLUME | O.VJP_POSE6, threads=1)
    np.testing.assert_allclose(gradient, volume, rtol=1e-12, atol=1e-14)
    stacked = np.concatenate([p for _, p in sorted(poses_all, key=lambda item: item[0])])
    np.testing.assert_allclose(stacked, pose, rtol=1e-12, atol=1e-15)
