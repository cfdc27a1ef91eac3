"""The CUDA transmission and objective kernels, through the C ABI via the host modules and the
Torch operators, against the golden vectors of the reference's exact Decimal oracles (with
the reference's budgets) and against the CPU oracle on the same inputs.

Exact where the arithmetic is shared: log transmission, the removed fraction and its inverse
(correctly rounded), the squared-error loss and seed, the Poisson seed.  Within the
reference's budgets where the FP32 exponential is involved (CUDA's expf and the C library's
may differ by an ULP or two): transmission within 4 ULPs, counts within 8, VJPs within
32 x 2^-24 of the summed magnitudes of their terms; the Poisson loss within 2e-15 relative.
"""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from dpt_b200.contracts import ContractError, NumericalError, TrialDomainError
from dpt_b200.objectives import (
    ObjectiveSpec,
    evaluate_objective,
    prepare_objective,
    reduce_objective_components,
)
from dpt_b200.torch import operators as ops
from dpt_b200.transmission import (
    GradientRangeError,
    TransmissionError,
    TransmissionOutputs,
    TransmissionSpec,
    optical_depth_from_removed,
    optical_depth_from_removed_vjp,
    prepare_transmission,
    transmission_vjp,
    transmit,
)
from oracle import pointwise as P
from test_oracle_pointwise import GOLDEN, ulps, within_forward_budget

pytestmark = pytest.mark.gpu
DEVICE = "cuda:0"


def dev(values, dtype=torch.float32):
    return torch.as_tensor(np.asarray(values), dtype=dtype, device=DEVICE).contiguous()


def host(tensor):
    return tensor.detach().cpu().numpy()


def test_forward_against_exact_rounding_and_oracle():
    depth, beam = GOLDEN["forward_depth"], GOLDEN["forward_beam"]
    n = depth.size
    ws = prepare_transmission(TransmissionSpec(beam="per-pixel"), max_pixels=n, device=DEVICE)
    outs = [torch.empty(n, device=DEVICE) for _ in range(4)]
    transmit(dev(depth), dev(beam), outputs=TransmissionOutputs(*outs), workspace=ws)
    t, counts, log_t, removed = (host(o) for o in outs)
    assert within_forward_budget(t, GOLDEN["forward_T"]).all()
    assert within_forward_budget(counts, GOLDEN["forward_counts"], counts=True).all()
    np.testing.assert_array_equal(log_t.view(np.uint32), GOLDEN["forward_log_T"].view(np.uint32))
    np.testing.assert_array_equal(removed.view(np.uint32), GOLDEN["forward_removed"].view(np.uint32))
    ot, oc, _, _ = P.transmit(depth, beam_mode=P.BEAM_PER_PIXEL, beam=beam)
    assert ulps(t, ot).max() <= 4 and ulps(counts, oc).max() <= 8


@pytest.mark.parametrize("mode", ["scalar", "device-scalar", "per-pixel"])
def test_beam_forms_and_single_outputs(mode):
    rng = np.random.default_rng(4)
    depth = rng.uniform(0, 30, 3000).astype(np.float32)
    n0 = np.float32(1234.5)
    beam_arg = {"scalar": float(n0), "device-scalar": dev([n0]), "per-pixel": dev(np.full(depth.size, n0))}[mode]
    ws = prepare_transmission(TransmissionSpec(beam=mode), max_pixels=depth.size, device=DEVICE)
    counts = torch.empty(depth.size, device=DEVICE)
    transmit(dev(depth), beam_arg, out_counts=counts, workspace=ws)
    _, expected, _, _ = P.transmit(depth, beam_mode=P.BEAM_SCALAR, beam_scalar=float(n0))
    assert ulps(host(counts), expected).max() <= 8
    assert (host(counts) > 0).all()


def test_small_range_identity_inverse_and_its_vjp():
    values = np.concatenate([np.array([0.0, -0.0], np.float32),
                             np.array([2.0**e for e in range(-149, -25)], np.float32)])
    ws = prepare_transmission(max_pixels=GOLDEN["inverse_delta"].size, device=DEVICE)
    removed = torch.empty(values.size, device=DEVICE)
    depth = torch.empty(values.size, device=DEVICE)
    transmit(dev(values), out_removed=removed, workspace=ws)
    optical_depth_from_removed(dev(values), out_L=depth, workspace=ws)
    expected = values.copy()
    expected[expected == 0] = 0.0
    np.testing.assert_array_equal(host(removed).view(np.uint32), expected.view(np.uint32))
    np.testing.assert_array_equal(host(depth).view(np.uint32), expected.view(np.uint32))
    delta = GOLDEN["inverse_delta"]
    out = torch.empty(delta.size, device=DEVICE)
    optical_depth_from_removed(dev(delta), out_L=out, workspace=ws)
    np.testing.assert_array_equal(host(out).view(np.uint32), GOLDEN["inverse_depth"].view(np.uint32))
    grad = torch.empty(delta.size, device=DEVICE)
    optical_depth_from_removed_vjp(dev(delta), dev(GOLDEN["inverse_seed"]), out_grad_delta=grad, workspace=ws)
    assert (np.abs(host(grad) - GOLDEN["inverse_grad"]) <= GOLDEN["inverse_budget"]).all()
    oracle_grad, _ = P.depth_from_removed_vjp(delta, GOLDEN["inverse_seed"])
    np.testing.assert_array_equal(host(grad), oracle_grad)


def test_vjp_against_exact_derivatives_and_oracle():
    g = GOLDEN
    n = g["vjp_depth"].size
    ws = prepare_transmission(TransmissionSpec(beam="per-pixel", active_beam=True), max_pixels=n, device=DEVICE)
    grad_L = torch.empty(n, device=DEVICE)
    grad_n0 = torch.empty(n, device=DEVICE)
    seeds = {k: dev(g[f"vjp_seed_{k}"]) for k in ("T", "counts", "log_T", "removed")}
    transmission_vjp(dev(g["vjp_depth"]), dev(g["vjp_beam"]), cotangent_T=seeds["T"],
                     cotangent_counts=seeds["counts"], cotangent_log_T=seeds["log_T"],
                     cotangent_removed=seeds["removed"], out_grad_L=grad_L, out_grad_n0=grad_n0, workspace=ws)
    assert (np.abs(host(grad_L) - g["vjp_grad_L"]) <= g["vjp_budget_L"]).all()
    assert (np.abs(host(grad_n0) - g["vjp_grad_n0"]) <= g["vjp_budget_n0"]).all()
    # shared device-scalar beam: the fixed FP64 tree
    shared_ws = prepare_transmission(TransmissionSpec(beam="device-scalar", active_beam=True), max_pixels=n,
                                     device=DEVICE)
    shared = torch.full((1,), 19.0, device=DEVICE)
    transmission_vjp(dev(g["vjp_depth"]), dev([7.0]), cotangent_counts=seeds["counts"], out_grad_L=grad_L,
                     out_grad_n0=shared, workspace=shared_ws)
    assert abs(float(shared[0]) - g["vjp_shared_n0"][0]) <= g["vjp_shared_budget"][0]
    _, oracle_shared, _ = P.transmit_vjp(g["vjp_depth"], beam_mode=P.BEAM_DEVICE_SCALAR,
                                         beam=np.array([7.0], np.float32), seed_counts=g["vjp_seed_counts"],
                                         beam_gradient="shared")
    assert abs(float(shared[0]) - float(oracle_shared[0])) <= g["vjp_shared_budget"][0]
    # without a count cotangent the shared gradient is an exact zero
    transmission_vjp(dev(g["vjp_depth"]), dev([7.0]), cotangent_T=seeds["T"], out_grad_n0=shared,
                     workspace=shared_ws)
    assert float(shared[0]) == 0.0


def test_count_free_per_pixel_beam_gradient_is_exact_zero():
    ws = prepare_transmission(TransmissionSpec(beam="per-pixel", active_beam=True), max_pixels=3, device=DEVICE)
    depth = dev([0.0, 0.25, 110.0])
    beam_grad = torch.full((3,), 19.0, device=DEVICE)
    depth_grad = torch.empty(3, device=DEVICE)
    seed = dev([2.0, -3.0, 4.0])
    transmission_vjp(depth, dev([1.0, 100.0, 1.0e30]), cotangent_T=seed, out_grad_L=depth_grad,
                     out_grad_n0=beam_grad, workspace=ws)
    assert (host(beam_grad) == 0).all()
    expected, _, _ = P.transmit_vjp(host(depth), seed_transmission=host(seed))
    assert ulps(host(depth_grad), expected).max() <= 4


def test_checked_calls_reject_inputs_and_leave_outputs_untouched():
    ws = prepare_transmission(max_pixels=8, device=DEVICE)
    out = torch.full((4,), 17.0, device=DEVICE)
    with pytest.raises(TransmissionError, match=r"L\[2\]=-1.0 violates finite_nonnegative"):
        transmit(dev([0.0, 1.0, -1.0, 2.0]), out_T=out, workspace=ws)
    assert (host(out) == 17).all()
    with pytest.raises(TransmissionError):  # the failed checkpoint stays set until cleared
        transmit(dev([0.0, 1.0, 1.0, 2.0]), out_T=out, workspace=ws)
    ws.clear_status()
    transmit(dev([0.0, 1.0, 1.0, 2.0]), out_T=out, workspace=ws)
    with pytest.raises(TransmissionError, match="delta"):
        optical_depth_from_removed(dev([0.5, 1.0]), out_L=torch.empty(2, device=DEVICE), workspace=ws)
    ws.clear_status()
    with pytest.raises(TransmissionError, match="overlaps"):
        depth = dev([0.5, 1.0])
        transmit(depth, out_T=depth, workspace=ws)
    with pytest.raises(TransmissionError, match="counts require"):
        transmit(dev([0.5]), out_counts=torch.empty(1, device=DEVICE), workspace=ws)
    # an unrepresentable gradient raises the range error
    wide = prepare_transmission(TransmissionSpec(beam="scalar"), max_pixels=1, device=DEVICE)
    with pytest.raises(GradientRangeError):
        transmission_vjp(dev([0.0]), 3.0e38, cotangent_counts=dev([3.0e38]), out_grad_L=torch.empty(1, device=DEVICE),
                         workspace=wide)


def test_unchecked_calls_are_asynchronous_until_the_checkpoint():
    ws = prepare_transmission(TransmissionSpec(beam="scalar"), max_pixels=1, device=DEVICE)
    grad = torch.empty(1, device=DEVICE)
    transmission_vjp(dev([0.0]), 3.0e38, cotangent_counts=dev([3.0e38]), out_grad_L=grad, workspace=ws,
                     validate=False)
    with pytest.raises(GradientRangeError):
        ws.consume_status()
    ws.check_status()  # consumed


def test_poisson_seams_in_fp64():
    g = GOLDEN
    ws = prepare_objective(ObjectiveSpec(kind="poisson", domain="counts", precision="float64"), max_pixels=1,
                           device=DEVICE)
    loss = torch.empty(1, dtype=torch.float64, device=DEVICE)
    seed = torch.empty(1, dtype=torch.float64, device=DEVICE)
    predictions = dev(g["poisson_prediction"], torch.float64)
    observations = dev(g["poisson_observation"])
    for k in range(predictions.numel()):
        evaluate_objective(predictions[k:k + 1], observations[k:k + 1], out_loss=loss, out_cotangent=seed,
                           workspace=ws)
        assert float(loss[0]) == pytest.approx(g["poisson_loss"][k], rel=2e-15, abs=0)
        assert float(seed[0]) == pytest.approx(g["poisson_derivative"][k], rel=4e-16, abs=0)


@pytest.mark.parametrize("precision", ["float32", "float64"])
@pytest.mark.parametrize("size", [255, 256, 257, 65537])
def test_multi_pixel_poisson_at_tree_boundaries(precision, size):
    dtype = torch.float64 if precision == "float64" else torch.float32
    ws = prepare_objective(ObjectiveSpec(kind="poisson", domain="counts", precision=precision), max_pixels=size,
                           device=DEVICE)
    i = np.arange(size)
    prediction = (1 + i % 13).astype(np.float64)
    observation = (i % 9).astype(np.float32)
    loss = torch.empty(1, dtype=torch.float64, device=DEVICE)
    seed = torch.empty(size, dtype=dtype, device=DEVICE)
    evaluate_objective(dev(prediction, dtype), dev(observation), out_loss=loss, out_cotangent=seed, workspace=ws)
    expected = math.fsum(GOLDEN["pattern_loss"][k % 117] for k in range(size))
    assert float(loss[0]) == pytest.approx(expected, rel=2e-15)
    reference = GOLDEN["pattern_derivative"][i % 117]
    np.testing.assert_allclose(host(seed), reference, rtol=2e-7 if precision == "float32" else 4e-16, atol=0)
    oracle_loss, oracle_seed, _ = P.objective(prediction.astype(host(seed).dtype), observation, poisson=True)
    np.testing.assert_array_equal(host(seed), oracle_seed)
    assert float(loss[0]) == pytest.approx(oracle_loss, rel=1e-15)


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_squared_error_weights_mask_mean_match_oracle_exactly(precision):
    dtype = torch.float64 if precision == "float64" else torch.float32
    rng = np.random.default_rng(9)
    n = 70001
    prediction = rng.normal(0, 10, n)
    observation = rng.normal(0, 10, n).astype(np.float32)
    weights = rng.uniform(0, 2, n).astype(np.float32)
    valid = (rng.uniform(size=n) > 0.2).astype(np.uint8)
    spec = ObjectiveSpec(reduction="mean", weighted=True, masked=True, precision=precision)
    ws = prepare_objective(spec, max_pixels=n, device=DEVICE)
    loss = torch.empty(1, dtype=torch.float64, device=DEVICE)
    seed = torch.empty(n, dtype=dtype, device=DEVICE)
    evaluate_objective(dev(prediction, dtype), dev(observation), out_loss=loss, out_cotangent=seed,
                       weights=dev(weights), valid=dev(valid, torch.uint8), workspace=ws)
    p = prediction.astype(np.float64 if precision == "float64" else np.float32)
    oracle_loss, oracle_seed, status = P.objective(p, observation, weights=weights, valid=valid, poisson=False,
                                                   normalisation=1.0 / n)
    assert status == 0
    np.testing.assert_array_equal(host(seed), oracle_seed)
    assert float(loss[0]) == oracle_loss
    assert (host(seed)[valid == 0] == 0).all()


@pytest.mark.parametrize("poisson", [False, True])
@pytest.mark.parametrize("checked", [False, True])
@pytest.mark.parametrize("value", [math.nan, math.inf, -math.inf])
def test_nonfinite_predictions_are_numerical_failures(poisson, checked, value):
    spec = ObjectiveSpec(kind="poisson" if poisson else "squared_error", domain="counts")
    ws = prepare_objective(spec, max_pixels=1, device=DEVICE)
    loss = torch.full((1,), 17.0, dtype=torch.float64, device=DEVICE)
    seed = torch.full((1,), 23.0, device=DEVICE)
    with pytest.raises(NumericalError) as error:
        evaluate_objective(dev([value]), torch.ones(1, device=DEVICE), out_loss=loss, out_cotangent=seed,
                           workspace=ws, validate=checked)
        ws.check_status()
    assert not isinstance(error.value, TrialDomainError)
    if checked:
        assert float(loss[0]) == 17.0 and float(seed[0]) == 23.0


def test_poisson_domain_and_invalid_observations():
    ws = prepare_objective(ObjectiveSpec(kind="poisson", domain="counts"), max_pixels=2, device=DEVICE)
    loss = torch.empty(1, dtype=torch.float64, device=DEVICE)
    with pytest.raises(TrialDomainError):
        evaluate_objective(dev([0.0, 1.0]), dev([2.0, 1.0]), out_loss=loss, workspace=ws)
    ws.clear_status()
    with pytest.raises(ContractError, match="integer counts"):
        evaluate_objective(dev([1.0, 1.0]), dev([1.5, 1.0]), out_loss=loss, workspace=ws)
    ws.clear_status()
    ws.validate_observation(dev([0.0, 3.0]))
    real = prepare_objective(ObjectiveSpec(kind="poisson", domain="counts", integer_counts=False), max_pixels=2,
                             device=DEVICE)
    evaluate_objective(dev([1.0, 1.0]), dev([1.5, 0.0]), out_loss=loss, workspace=real)
    assert float(loss[0]) == pytest.approx(1.0 - 1.5 + 1.5 * math.log(1.5) + 1.0, rel=1e-15)


def test_component_reduction_is_fixed_order():
    values = np.random.default_rng(2).normal(size=300000)
    ws = prepare_objective(ObjectiveSpec(), max_pixels=values.size, device=DEVICE)
    out = torch.empty(1, dtype=torch.float64, device=DEVICE)
    reduce_objective_components(dev(values, torch.float64), out_loss=out, workspace=ws)
    assert float(out[0]) == P.tree_sum(values)
    reduce_objective_components(dev(values[:0], torch.float64), out_loss=out, workspace=ws)
    assert float(out[0]) == 0.0


@pytest.mark.parametrize("output", ["transmission", "counts", "log_transmission", "removed"])
def test_torch_transmit_forward_and_backward(output):
    rng = np.random.default_rng(12)
    depth_np = rng.uniform(0, 6, (48, 40)).astype(np.float32)
    beam_np = rng.uniform(10, 1000, (48, 40)).astype(np.float32)
    ws = prepare_transmission(TransmissionSpec(beam="per-pixel", active_beam=True), max_pixels=depth_np.size,
                              device=DEVICE)
    depth = dev(depth_np).requires_grad_()
    beam = dev(beam_np).requires_grad_()
    image = ops.transmit(depth, beam, output=output, workspace=ws)
    assert image.shape == depth.shape and image.dtype == torch.float32
    seed_np = rng.uniform(-1, 1, depth_np.shape).astype(np.float32)
    image.backward(dev(seed_np))
    name = {"transmission": "seed_transmission", "counts": "seed_counts", "log_transmission": "seed_log",
            "removed": "seed_removed"}[output]
    grad_L, grad_beam, _ = P.transmit_vjp(depth_np, beam_mode=P.BEAM_PER_PIXEL, beam=beam_np, **{name: seed_np},
                                          beam_gradient="per-pixel")
    assert ulps(host(depth.grad).reshape(-1), grad_L).max() <= 4
    assert ulps(host(beam.grad).reshape(-1), grad_beam).max() <= 4


def test_torch_transmit_shared_beam_and_fixed_inputs():
    rng = np.random.default_rng(13)
    depth_np = rng.uniform(0, 3, 5000).astype(np.float32)
    ws = prepare_transmission(TransmissionSpec(beam="device-scalar", active_beam=True), max_pixels=5000,
                              device=DEVICE)
    depth = dev(depth_np).requires_grad_()
    beam = dev([250.0]).requires_grad_()
    counts = ops.transmit(depth, beam, output="counts", workspace=ws)
    counts.sum().backward()
    _, shared, _ = P.transmit_vjp(depth_np, beam_mode=P.BEAM_DEVICE_SCALAR, beam=np.array([250.0], np.float32),
                                  seed_counts=np.ones(5000, np.float32), beam_gradient="shared")
    assert float(beam.grad[0]) == pytest.approx(float(shared[0]), rel=1e-6)
    fixed = prepare_transmission(TransmissionSpec(active_L=False), max_pixels=4, device=DEVICE)
    with pytest.raises(ContractError, match="declared fixed"):
        ops.transmit(dev([1.0]).requires_grad_(), workspace=fixed)


@pytest.mark.parametrize("precision", ["float32", "float64"])
@pytest.mark.parametrize("kind", ["squared_error", "poisson"])
def test_torch_objective_forward_and_backward(precision, kind):
    dtype = torch.float64 if precision == "float64" else torch.float32
    rng = np.random.default_rng(14)
    shape = (30, 33)
    prediction_np = rng.uniform(0.5, 20, shape)
    observation_np = rng.integers(0, 25, shape).astype(np.float32)
    weights_np = rng.uniform(0, 1, shape).astype(np.float32)
    spec = ObjectiveSpec(kind=kind, domain="counts", weighted=True, precision=precision, reduction="mean")
    ws = prepare_objective(spec, max_pixels=prediction_np.size, device=DEVICE)
    prediction = dev(prediction_np, dtype).requires_grad_()
    loss = ops.objective(prediction, dev(observation_np), weights=dev(weights_np), workspace=ws)
    assert loss.dtype == torch.float64 and loss.shape == ()
    p = prediction_np.astype(np.float64 if precision == "float64" else np.float32).reshape(-1)
    oracle_loss, _, _ = P.objective(p, observation_np, weights=weights_np, poisson=kind == "poisson",
                                    normalisation=1.0 / p.size)
    assert float(loss.detach()) == pytest.approx(oracle_loss, rel=1e-15)
    (3.0 * loss).backward()
    _, oracle_seed, _ = P.objective(p, observation_np, weights=weights_np, poisson=kind == "poisson",
                                    wide=True, normalisation=1.0 / p.size, seed_scale=3.0)
    np.testing.assert_array_equal(host(prediction.grad).reshape(-1), oracle_seed)


def test_torch_objective_zero_cotangent_and_first_order_only():
    ws = prepare_objective(ObjectiveSpec(), max_pixels=4, device=DEVICE)
    prediction = dev([1.0, 2.0]).requires_grad_()
    loss = ops.objective(prediction, dev([0.0, 0.0]), workspace=ws)
    (0.0 * loss).backward()
    assert (host(prediction.grad) == 0).all()
    prediction.grad = None
    loss = ops.objective(prediction, dev([0.0, 0.0]), workspace=ws)
    with pytest.raises(ContractError, match="first-order"):
        torch.autograd.grad(loss, prediction, create_graph=True)
    with pytest.raises(ContractError, match="fixed"):
        ops.objective(prediction, dev([0.0, 0.0]).requires_grad_(), workspace=ws)


def test_full_size_round_trip_and_determinism():
    """2^26 pixels: removed + T within 2^-22 of one, L -> removed -> L round trip, and a
    repeated objective gives the same FP64 bits."""
    n = 1 << 26
    generator = torch.Generator(device=DEVICE).manual_seed(5)
    depth = torch.rand(n, device=DEVICE, generator=generator) * 8
    ws = prepare_transmission(max_pixels=n, device=DEVICE)
    t = torch.empty(n, device=DEVICE)
    removed = torch.empty(n, device=DEVICE)
    transmit(depth, out_T=t, out_removed=removed, workspace=ws)
    assert float((t.double() + removed.double() - 1).abs().max()) <= 2.0**-22
    back = torch.empty(n, device=DEVICE)
    small = depth.clamp(max=0.4)  # removed <= 1/3, the round trip is well conditioned
    transmit(small, out_removed=removed, workspace=ws)
    optical_depth_from_removed(removed, out_L=back, workspace=ws)
    assert float(((back - small).abs() / small.clamp(min=1e-30)).max()) <= 4 * 2.0**-24
    objective_ws = prepare_objective(ObjectiveSpec(kind="poisson", domain="counts"), max_pixels=n, device=DEVICE)
    observation = torch.poisson(t * 50, generator=generator)
    prediction = t * 50 + 1e-3
    first = torch.empty(1, dtype=torch.float64, device=DEVICE)
    second = torch.empty(1, dtype=torch.float64, device=DEVICE)
    evaluate_objective(prediction, observation, out_loss=first, workspace=objective_ws)
    evaluate_objective(prediction, observation, out_loss=second, workspace=objective_ws)
    assert float(first[0]) == float(second[0])


@pytest.mark.parametrize("offset", [0, 1, 3])
@pytest.mark.parametrize("size", [1, 5, 4095, 4097, 70003])
def test_ragged_sizes_and_unaligned_views(offset, size):
    """Tails that are not whole vector groups and views whose pointers are not 16-byte aligned
    take the element-wise path and give the same bits as the aligned one."""
    rng = np.random.default_rng(size + offset)
    depth_np = rng.uniform(0, 5, size).astype(np.float32)
    seed_np = rng.uniform(-1, 1, size).astype(np.float32)
    storage = torch.zeros(size + 8, device=DEVICE)
    storage[offset:offset + size] = dev(depth_np)
    depth = storage[offset:offset + size]
    outputs = torch.full((4, size + 8), 7.0, device=DEVICE)
    views = [outputs[i, offset:offset + size] for i in range(4)]
    ws = prepare_transmission(TransmissionSpec(beam="scalar"), max_pixels=size, device=DEVICE)
    transmit(depth, 3.0, outputs=TransmissionOutputs(*views), workspace=ws)
    aligned = [torch.empty(size, device=DEVICE) for _ in range(4)]
    transmit(dev(depth_np), 3.0, outputs=TransmissionOutputs(*aligned), workspace=ws)
    for view, reference in zip(views, aligned):
        np.testing.assert_array_equal(host(view), host(reference))
    assert (host(outputs[:, :offset]) == 7).all() and (host(outputs[:, offset + size:]) == 7).all()
    grad_storage = torch.full((size + 8,), 5.0, device=DEVICE)
    seed_storage = torch.zeros(size + 8, device=DEVICE)
    seed_storage[offset:offset + size] = dev(seed_np)
    transmission_vjp(depth, 3.0, cotangent_removed=seed_storage[offset:offset + size],
                     out_grad_L=grad_storage[offset:offset + size], workspace=ws)
    expected, _, _ = P.transmit_vjp(depth_np, seed_removed=seed_np)
    assert ulps(host(grad_storage[offset:offset + size]), expected).max() <= 4
    assert float(grad_storage[-1]) == 5.0
    objective_ws = prepare_objective(ObjectiveSpec(weighted=True), max_pixels=size, device=DEVICE)
    observation_np = rng.normal(size=size).astype(np.float32)
    weights_np = rng.uniform(0, 1, size).astype(np.float32)
    obs_storage = torch.zeros(size + 8, device=DEVICE)
    obs_storage[offset:offset + size] = dev(observation_np)
    loss = torch.empty(1, dtype=torch.float64, device=DEVICE)
    cot = torch.empty(size + 8, device=DEVICE)
    evaluate_objective(depth, obs_storage[offset:offset + size], out_loss=loss, out_cotangent=cot[offset:offset + size],
                       weights=dev(weights_np), workspace=objective_ws)
    oracle_loss, oracle_seed, _ = P.objective(depth_np, observation_np, weights=weights_np, poisson=False)
    assert float(loss[0]) == oracle_loss
    np.testing.assert_array_equal(host(cot[offset:offset + size]), oracle_seed)
