"""Serving: admission and tuning logic on the CPU; on the GPU, every request's result is
the same alone and inside a concurrent mix (forward images bit-exact, gradients within
the atomic-order tolerance), graph replays match first runs, and the budget holds."""

from __future__ import annotations

import math
import random

import numpy as np
import pytest

from dpt_b200.contracts import ContractError
from dpt_b200.serving import Admission, ProjectionRequest, TileTuner, percentile


def test_admission_first_fit_and_budget():
    admission = Admission(100, lookahead=4)
    for name, size in (("a", 60), ("b", 50), ("c", 30), ("d", 20)):
        admission.offer(name, size)
    started = admission.take(4)
    assert [name for name, _ in started] == ["a", "c"]  # b waits for memory, c backfills
    assert admission.in_use == 90
    admission.release(60)
    assert [name for name, _ in admission.take(4)] == ["b", "d"]  # 30 + 50 + 20 = 100 fits exactly
    assert admission.in_use == 100 and not admission.waiting
    with pytest.raises(ContractError):
        admission.offer("huge", 101)
    with pytest.raises(ContractError):
        Admission(0)


def test_admission_respects_slot_count_and_order():
    admission = Admission(1000)
    for k in range(10):
        admission.offer(k, 10)
    assert [k for k, _ in admission.take(3)] == [0, 1, 2]
    assert [k for k, _ in admission.take(2)] == [3, 4]
    assert admission.in_use == 50


def test_tuner_keeps_the_fastest_tile_by_its_best_time_and_the_default_within_the_margin():
    calls = []
    noise = iter([0.0, 0.5, 0.2] * 8)

    def run(cols):
        calls.append(cols)
        return {8: 3.0, 16: 2.0, 32: 1.0, 64: 4.0}[cols] + next(noise)

    tuner = TileTuner(repeats=3, margin=0.03)
    assert tuner.choose("k", run) == 32
    assert tuner.choose("k", run) == 32
    assert sorted(calls) == sorted([8, 16, 32, 64] * 3)
    assert tuner.timings["k"] == {8: 3.0, 16: 2.0, 32: 1.0, 64: 4.0}

    # 2 % faster than the default is within the margin: the default stays
    close = TileTuner(repeats=1, margin=0.03)
    assert close.choose("c", lambda cols: {8: 3.0, 16: 1.0, 32: 0.98, 64: 4.0}[cols]) == 16
    assert close.choose("d", lambda cols: {8: 3.0, 16: 1.0, 32: 0.9, 64: 4.0}[cols]) == 32


def test_percentiles_and_request_contracts():
    values = list(range(1, 101))
    assert percentile(values, 50) == 50 and percentile(values, 99) == 99 and percentile(values, 100) == 100
    with pytest.raises(ContractError):
        ProjectionRequest("v", None, 0)
    with pytest.raises(ContractError):
        ProjectionRequest("v", None, 8, kind="both")


# ------------------------------------------------------------------- GPU


def _scenes():
    from dpt_b200.geometry import ConeBeamIntrinsics
    from dpt_b200.phantoms import centred_grid, ellipsoid_phantom

    out = {}
    for name, shape, spacing in (("small", (20, 24, 28), 1.0), ("mid", (40, 36, 32), 0.8)):
        grid = centred_grid(shape, (spacing,) * 3)
        values, _ = ellipsoid_phantom(grid, seed=len(name), count=3)
        out[name] = (grid, values)
    return out, ConeBeamIntrinsics


def _requests(seed: int = 3, count: int = 14):
    from dpt_b200.serving import ProjectionRequest

    scenes, intrinsics_type = _scenes()
    rng = random.Random(seed)
    requests = []
    for _ in range(count):
        name = rng.choice(sorted(scenes))
        views = rng.choice((1, 2, 5))
        detector = rng.choice((16, 24, 40))
        intrinsics = intrinsics_type(120.0, 200.0, (detector, detector), (1.6, 1.6))
        geometry = intrinsics.batch(tuple(2 * math.pi * k / views + 0.3 for k in range(views)))
        kind = rng.choice(("forward", "forward", "volume", "pose"))
        target = np.full((views, detector, detector), 0.05, dtype=np.float32)
        tangent = np.asarray([0.2, -0.1, 0.05, 0.01, 0.0, -0.02]) if kind == "pose" else None
        requests.append(ProjectionRequest(name, geometry, rng.choice((32, 48)), kind, target, tangent))
    return scenes, requests


@pytest.mark.gpu
@pytest.mark.parametrize("graphs,priorities", [(False, False), (True, False), (True, True)])
def test_results_are_the_same_alone_and_in_the_mix(graphs, priorities):
    from dpt_b200.serving import ProjectionServer

    scenes, requests = _requests()
    with ProjectionServer("cuda:0", slots=4, graphs=graphs, autotune=graphs, priorities=priorities,
                          exclusive_samples=1 << 18) as server:
        for name, (grid, values) in scenes.items():
            server.add_volume(name, grid, values)
        alone = [server.run_alone(request) for request in requests]
        futures = [server.submit(request) for request in requests + requests]
        mixed = [future.result(timeout=300) for future in futures]
    for k, request in enumerate(requests + requests):
        a, m = alone[k % len(requests)], mixed[k]
        np.testing.assert_array_equal(m.image.cpu().numpy(), a.image.cpu().numpy())
        if request.kind == "volume":
            va, vm = a.volume_gradient.cpu().numpy(), m.volume_gradient.cpu().numpy()
            assert np.linalg.norm(va - vm) <= 1e-6 * np.linalg.norm(va)
        if request.kind == "pose":
            np.testing.assert_allclose(m.pose_gradient.cpu().numpy(), a.pose_gradient.cpu().numpy(),
                                       rtol=1e-10, atol=1e-13)
        if request.kind != "forward":
            assert m.loss == pytest.approx(a.loss, rel=1e-12)
        assert m.latency > 0


@pytest.mark.gpu
def test_chained_requests_match_the_same_requests_alone():
    """run_chained (the launch sequences back to back, one synchronisation) returns what
    run_alone returns for each request: its own readback buffers, no shared staging."""
    from dpt_b200.serving import ProjectionServer

    scenes, requests = _requests(seed=5, count=10)
    with ProjectionServer("cuda:0", slots=1, graphs=False, autotune=False) as server:
        for name, (grid, values) in scenes.items():
            server.add_volume(name, grid, values)
        alone = [server.run_alone(request) for request in requests]
        chained = server.run_chained(requests)
    for request, a, c in zip(requests, alone, chained, strict=True):
        np.testing.assert_array_equal(c.image.cpu().numpy(), a.image.cpu().numpy())
        if request.kind == "volume":
            va, vc = a.volume_gradient.cpu().numpy(), c.volume_gradient.cpu().numpy()
            assert np.linalg.norm(va - vc) <= 1e-6 * np.linalg.norm(va)
        if request.kind == "pose":
            np.testing.assert_allclose(c.pose_gradient.cpu().numpy(), a.pose_gradient.cpu().numpy(),
                                       rtol=1e-10, atol=1e-13)
        if request.kind != "forward":
            assert c.loss == pytest.approx(a.loss, rel=1e-12)


@pytest.mark.gpu
def test_budget_limits_concurrency():
    from dpt_b200.serving import ProjectionServer

    scenes, requests = _requests(seed=5, count=6)
    with ProjectionServer("cuda:0", slots=4, graphs=False, autotune=False) as server:
        for name, (grid, values) in scenes.items():
            server.add_volume(name, grid, values)
        largest = max(server.request_bytes(r) for r in requests)
        server.admission.budget = largest  # one request at a time fits
        results = [f.result(timeout=300) for f in [server.submit(r) for r in requests]]
    assert len(results) == len(requests)
    assert server.admission.peak <= largest
    assert server.admission.in_use == 0


@pytest.mark.gpu
def test_shared_field_copies_and_scratch_pool_match_private_workspaces():
    import torch

    from dpt_b200.plan import plan_rays
    from dpt_b200.projection import FieldCopies, ProjectionSpec, ProjectionWorkspace, ScratchPool

    scenes, intrinsics_type = _scenes()
    grid, values = scenes["mid"]
    field = torch.tensor(values, device="cuda:0")
    copies, pool = FieldCopies(), ScratchPool("cuda:0")
    geometries = [intrinsics_type(120.0, 200.0, (n, n), (1.6, 1.6)).batch((0.1 * n, 0.2 * n)) for n in (16, 24)]
    for sampling in ("float32", "compensated"):
        spec = ProjectionSpec(40, sampling_precision=sampling, active_volume=True)
        private = [ProjectionWorkspace(plan_rays(grid, g), spec, "cuda:0") for g in geometries]
        shared = [ProjectionWorkspace(plan_rays(grid, g), spec, "cuda:0", copies=copies, pool=pool)
                  for g in geometries]
        poses = torch.tensor((1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0, 0, 0, 0), dtype=torch.float64, device="cuda:0")
        side = torch.cuda.Stream()
        for round_ in range(2):
            if round_ == 1:
                field.mul_(1.5)  # in-place change: every copy must be rewritten
            for p, s in zip(private, shared, strict=True):
                poses_v = poses.expand(p.views, 12).contiguous()
                expected = p.forward(field, poses_v)
                with torch.cuda.stream(side):  # the shared copy is written on another stream
                    side.wait_stream(torch.cuda.current_stream())
                    got = s.forward(field, poses_v)
                torch.cuda.current_stream().wait_stream(side)
                torch.testing.assert_close(got, expected, rtol=0, atol=0)
                cot = torch.full_like(expected, 0.25)
                g_expected, _ = p.vjp(field, poses_v, cot, volume=True, pose=None)
                g_got, _ = s.vjp(field, poses_v, cot, volume=True, pose=None)
                assert torch.linalg.norm(g_got - g_expected) <= 1e-6 * torch.linalg.norm(g_expected)
        assert copies.bytes() > 0


def test_admission_holds_back_ineligible_items_without_blocking_the_rest():
    admission = Admission(1000, lookahead=8)
    for name in ("big1", "small1", "big2", "small2"):
        admission.offer(name, 10)
    # one large item may start: the second waits, the small ones pass it
    started = [0]

    def eligible(name):
        if name.startswith("big"):
            if started[0]:
                return False
            started[0] += 1
        return True

    assert [name for name, _ in admission.take(4, eligible)] == ["big1", "small1", "small2"]
    assert [name for name, _ in admission.waiting] == ["big2"]
    assert [name for name, _ in admission.take(4)] == ["big2"]


def test_admission_take_matching_fills_a_pack_in_arrival_order_within_the_budget():
    admission = Admission(100, lookahead=2)
    for name, size in (("a1", 10), ("b1", 10), ("a2", 70), ("a3", 20), ("b2", 5), ("a4", 30)):
        admission.offer(name, size)
    first = admission.take(1)
    assert [name for name, _ in first] == ["a1"]
    # the whole queue is scanned (beyond the look-ahead); a2 does not fit beside a3 and a4
    companions = admission.take_matching(lambda name: name.startswith("a"), limit=8)
    assert [name for name, _ in companions] == ["a2", "a3"]
    assert admission.in_use == 100
    assert [name for name, _ in admission.waiting] == ["b1", "b2", "a4"]
    admission.release(100)
    assert [name for name, _ in admission.take_matching(lambda name: True, limit=2)] == ["b1", "b2"]


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["float32", "bfloat16"])
def test_packed_small_forward_requests_match_each_alone(storage):
    """A burst of small forward requests on one slot runs as packed launches; every image is
    the one the same request gives alone, and the gradient requests in the burst are unchanged."""
    from dpt_b200.serving import ProjectionServer

    scenes, requests = _requests(seed=9, count=24)
    with ProjectionServer("cuda:0", slots=1, graphs=False, autotune=True, pack_min=2) as server:
        for name, (grid, values) in scenes.items():
            server.add_volume(name, grid, values, storage=storage)
        alone = [server.run_alone(request) for request in requests]
        futures = [server.submit(request) for request in requests + requests]
        mixed = [future.result(timeout=300) for future in futures]
        assert server.packs > 0 and server.packed_requests >= 2 * server.packs
        assert server.admission.in_use == 0
    for k, request in enumerate(requests + requests):
        a, m = alone[k % len(requests)], mixed[k]
        np.testing.assert_array_equal(m.image.cpu().numpy(), a.image.cpu().numpy())
        if request.kind == "volume":
            va, vm = a.volume_gradient.float().cpu().numpy(), m.volume_gradient.float().cpu().numpy()
            assert np.linalg.norm(va - vm) <= 1e-6 * np.linalg.norm(va)
        if request.kind == "pose":
            np.testing.assert_allclose(m.pose_gradient.cpu().numpy(), a.pose_gradient.cpu().numpy(),
                                       rtol=1e-10, atol=1e-13)


def _items(*specs):
    """(name, pack_class, large, medium) -> simple request stand-ins."""
    from types import SimpleNamespace

    return [SimpleNamespace(name=n, pack_class=c, large=lg, medium=md) for n, c, lg, md in specs]


def test_launch_policy_packs_the_oldest_due_class_and_holds_it_from_the_slots():
    from dpt_b200.serving import LaunchPolicy

    admission = Admission(1000)
    items = _items(("a1", "A", False, False), ("b1", "B", False, False), ("a2", "A", False, False),
                   ("x", None, False, False), ("b2", "B", False, False), ("b3", "B", False, False))
    for item in items:
        admission.offer(item, 10)
    policy = LaunchPolicy(pack_min=3, max_pack=64, lane=True)
    # class B is due (3 waiting), A is not: the lane takes all of B, the oldest due class
    assert policy.startable(admission, lane_free=True, any_slot_free=False, large_running=0)
    assert [i.name for i in policy.take_pack(admission)] == ["b1", "b2", "b3"]
    assert policy.take_pack(admission) == []
    taken, large = policy.take_singles(admission, free_slots=4, large_running=0)
    assert [i.name for i in taken] == ["a1", "a2", "x"] and large == 0


def test_launch_policy_keeps_a_due_class_for_the_busy_lane_and_sleeps_when_nothing_can_start():
    from dpt_b200.serving import LaunchPolicy

    admission = Admission(1000)
    for item in _items(("a1", "A", False, False), ("a2", "A", False, False)):
        admission.offer(item, 10)
    policy = LaunchPolicy(pack_min=2, max_pack=64, lane=True)
    # the lane is busy: the slots must not take the due class, so there is nothing to start
    assert not policy.startable(admission, lane_free=False, any_slot_free=True, large_running=0)
    assert policy.take_singles(admission, free_slots=4, large_running=0) == ([], 0)
    # without a lane the same items are ordinary requests
    plain = LaunchPolicy(pack_min=2, max_pack=64, lane=False)
    assert plain.startable(admission, lane_free=False, any_slot_free=True, large_running=0)
    assert plain.take_pack(admission) == []
    assert [i.name for i in plain.take_singles(admission, 4, 0)[0]] == ["a1", "a2"]


def test_launch_policy_runs_large_requests_alone_with_only_small_ones_beside():
    from dpt_b200.serving import LaunchPolicy

    admission = Admission(1000)
    for item in _items(("L1", None, True, False), ("m1", None, False, True), ("L2", None, True, False),
                       ("s1", None, False, False)):
        admission.offer(item, 10)
    policy = LaunchPolicy(pack_min=8, max_pack=64, lane=True)
    taken, large = policy.take_singles(admission, free_slots=4, large_running=0)
    assert [i.name for i in taken] == ["L1", "s1"] and large == 1  # m1 and L2 wait for L1
    assert not policy.startable(admission, lane_free=True, any_slot_free=True, large_running=1)
    taken, large = policy.take_singles(admission, free_slots=4, large_running=0)
    assert [i.name for i in taken] == ["m1", "L2"] and large == 1  # m1 started before L2 in order


def test_launch_policy_pack_respects_the_memory_budget():
    from dpt_b200.serving import LaunchPolicy

    admission = Admission(25)
    for item in _items(("a1", "A", False, False), ("a2", "A", False, False), ("a3", "A", False, False)):
        admission.offer(item, 10)
    policy = LaunchPolicy(pack_min=3, max_pack=64, lane=True)
    # due, but only two of the three fit: the pack takes what fits, the rest waits
    assert [i.name for i in policy.take_pack(admission)] == ["a1", "a2"]
    assert admission.in_use == 20 and [i.name for i, _ in admission.waiting] == ["a3"]
    # one waiting item is no longer a due pack; it may go to a slot once memory is released
    assert policy.take_singles(admission, free_slots=1, large_running=0) == ([], 0)
    admission.release(20)
    assert [i.name for i in policy.take_singles(admission, free_slots=1, large_running=0)[0]] == ["a3"]
