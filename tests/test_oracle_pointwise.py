"""The CPU pointwise oracle (transmission and objectives) pinned to the reference's exact
Decimal oracles through the committed golden vectors (``golden/make_pointwise_golden.py``),
with the reference's own error budgets: forward values within 4 binary32 ULPs (8 for counts,
1 in the subnormal range) of the correctly rounded value, the removed fraction and its inverse
correctly rounded, VJPs within 32 x 2^-24 of the summed magnitudes of their terms, the Poisson
loss within 2e-15 and its FP64 seed within 4e-16 (relative).  Oracle-only: no GPU.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from oracle import pointwise as P

GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "pointwise.npz")
MIN_NORMAL = float(np.finfo(np.float32).tiny)


def ulps(actual, expected) -> np.ndarray:
    """Binary32 steps between two arrays; signed zeros are zero apart."""
    def ordered(values):
        bits = np.asarray(values, dtype=np.float32).view(np.uint32).astype(np.int64)
        return np.where(bits >> 31, 0x80000000 - (bits & 0x7FFFFFFF), 0x80000000 + bits)
    return np.abs(ordered(actual) - ordered(expected))


def within_forward_budget(actual, expected, *, counts: bool = False) -> np.ndarray:
    allowed = np.where(np.abs(expected) < MIN_NORMAL, 1, 8 if counts else 4)
    return ulps(actual, expected) <= allowed


def test_forward_against_exact_rounding():
    depth, beam = GOLDEN["forward_depth"], GOLDEN["forward_beam"]
    t, _, log_t, removed = P.transmit(depth)
    _, counts, _, _ = P.transmit(depth, beam_mode=P.BEAM_PER_PIXEL, beam=beam)
    assert within_forward_budget(t, GOLDEN["forward_T"]).all()
    assert within_forward_budget(counts, GOLDEN["forward_counts"], counts=True).all()
    np.testing.assert_array_equal(log_t.view(np.uint32), GOLDEN["forward_log_T"].view(np.uint32))
    # the removed fraction is correctly rounded (the reference's own bit-exact claim)
    np.testing.assert_array_equal(removed.view(np.uint32), GOLDEN["forward_removed"].view(np.uint32))
    # the deep tail keeps the count product in range: exp(-110) underflows FP32, 1e30 T does not
    deep = np.array([110.0, 200.0], np.float32)
    t, counts, _, _ = P.transmit(deep, beam_mode=P.BEAM_SCALAR, beam_scalar=1.0e30)
    assert t[0] == 0 and counts[0] > 0


def test_small_range_identity_and_positive_zero():
    values = np.concatenate([np.array([0.0, -0.0], np.float32),
                             np.array([2.0**e for e in range(-149, -25)], np.float32)])
    _, _, _, removed = P.transmit(values)
    depth = P.depth_from_removed(values)
    expected = values.copy()
    expected[expected == 0] = 0.0
    np.testing.assert_array_equal(removed.view(np.uint32), expected.view(np.uint32))
    np.testing.assert_array_equal(depth.view(np.uint32), expected.view(np.uint32))


def test_inverse_against_exact_rounding():
    delta = GOLDEN["inverse_delta"]
    depth = P.depth_from_removed(delta)
    np.testing.assert_array_equal(depth.view(np.uint32), GOLDEN["inverse_depth"].view(np.uint32))
    grad, status = P.depth_from_removed_vjp(delta, GOLDEN["inverse_seed"])
    assert status == 0
    assert (np.abs(grad - GOLDEN["inverse_grad"]) <= GOLDEN["inverse_budget"]).all()


def test_vjp_against_exact_derivatives():
    g = GOLDEN
    grad, pixels, status = P.transmit_vjp(
        g["vjp_depth"], beam_mode=P.BEAM_PER_PIXEL, beam=g["vjp_beam"], seed_transmission=g["vjp_seed_T"],
        seed_counts=g["vjp_seed_counts"], seed_log=g["vjp_seed_log_T"], seed_removed=g["vjp_seed_removed"],
        beam_gradient="per-pixel")
    assert status == 0
    assert (np.abs(grad - g["vjp_grad_L"]) <= g["vjp_budget_L"]).all()
    assert (np.abs(pixels - g["vjp_grad_n0"]) <= g["vjp_budget_n0"]).all()
    _, shared, status = P.transmit_vjp(g["vjp_depth"], beam_mode=P.BEAM_DEVICE_SCALAR,
                                       beam=np.array([7.0], np.float32), seed_counts=g["vjp_seed_counts"],
                                       beam_gradient="shared")
    assert status == 0
    assert abs(float(shared[0]) - g["vjp_shared_n0"][0]) <= g["vjp_shared_budget"][0]


def test_vjp_boundary_identities():
    zero = np.zeros(1, np.float32)
    one = np.ones(1, np.float32)
    grad, _, _ = P.transmit_vjp(zero, seed_transmission=one)
    assert grad[0] == -1
    grad, _, _ = P.transmit_vjp(zero, seed_removed=one)
    assert grad[0] == 1
    grad, _, _ = P.transmit_vjp(zero, seed_log=one)
    assert grad[0] == -1
    _, beam, _ = P.transmit_vjp(zero, beam_mode=P.BEAM_PER_PIXEL, beam=zero, seed_counts=one,
                                beam_gradient="per-pixel")
    assert beam[0] == 1
    # an FP32-overflowing derivative sets the range bit
    _, _, status = P.transmit_vjp(zero, beam_mode=P.BEAM_SCALAR, beam_scalar=3.0e38,
                                  seed_counts=np.array([3.0e38], np.float32))
    assert status == 2


def test_poisson_loss_and_seed_across_cancellation_seams():
    g = GOLDEN
    for mu, y, loss_ref, deriv_ref in zip(g["poisson_prediction"], g["poisson_observation"], g["poisson_loss"],
                                          g["poisson_derivative"]):
        loss, seed, status = P.objective(np.array([mu]), np.array([y], np.float32), poisson=True)
        assert status == 0
        assert loss == pytest.approx(loss_ref, rel=2e-15, abs=0)
        assert seed[0] == pytest.approx(deriv_ref, rel=4e-16, abs=0)


@pytest.mark.parametrize("precision", ["float32", "float64"])
@pytest.mark.parametrize("size", [255, 256, 257, 65537])
def test_multi_pixel_poisson_at_tree_boundaries(precision, size):
    dtype = np.float64 if precision == "float64" else np.float32
    i = np.arange(size)
    prediction = (1 + i % 13).astype(dtype)
    observation = (i % 9).astype(np.float32)
    loss, seed, status = P.objective(prediction, observation, poisson=True)
    assert status == 0
    expected = math.fsum(GOLDEN["pattern_loss"][k % 117] for k in range(size))
    assert loss == pytest.approx(expected, rel=2e-15)
    reference = GOLDEN["pattern_derivative"][i % 117].astype(dtype)
    np.testing.assert_allclose(seed, reference, rtol=2e-7 if precision == "float32" else 4e-16, atol=0)


def test_squared_error_is_exact_arithmetic():
    g = GOLDEN
    loss, seed, status = P.objective(g["squared_prediction"], g["squared_observation"], poisson=False)
    assert status == 0
    np.testing.assert_array_equal(seed, g["squared_derivative"])
    assert loss == pytest.approx(math.fsum(g["squared_loss"]), rel=1e-14)


def test_weights_mask_mean_and_statuses():
    rng = np.random.default_rng(3)
    n = 1000
    prediction = rng.uniform(1, 5, n).astype(np.float32)
    observation = rng.integers(0, 6, n).astype(np.float32)
    weights = rng.uniform(0, 2, n).astype(np.float32)
    valid = (rng.uniform(size=n) > 0.3).astype(np.uint8)
    loss, seed, status = P.objective(prediction, observation, weights=weights, valid=valid, poisson=True,
                                     normalisation=1.0 / n)
    assert status == 0
    active = valid == 1
    mu, y, w = prediction.astype(np.float64), observation.astype(np.float64), weights.astype(np.float64) / n
    terms = np.where(y > 0, mu - y + y * np.log(np.where(y > 0, y, 1) / mu), mu)
    assert loss == pytest.approx(float(np.sum((w * terms)[active])), rel=1e-12)
    assert (seed[~active] == 0).all()
    np.testing.assert_allclose(seed[active], ((w * (mu - y) / mu)[active]).astype(np.float32), rtol=1e-6)
    # invalid fixed inputs, domain and range bits
    assert P.objective_check(None, np.array([1.5], np.float32), poisson=True) == 1
    assert P.objective_check(None, np.array([1.5], np.float32), poisson=True, integer_counts=False) == 0
    assert P.objective_check(None, np.array([1.0], np.float32), valid=np.array([2]), poisson=False) == 1
    assert P.objective_check(np.array([0.0], np.float32), np.array([2.0], np.float32), poisson=True) == 8
    assert P.objective_check(np.array([-1.0], np.float32), np.array([0.0], np.float32), poisson=True) == 8
    assert P.objective_check(np.array([np.nan], np.float32), np.array([1.0], np.float32), poisson=False) == 2
    _, _, status = P.objective(np.array([3.0e38], np.float32), np.array([-3.0e38], np.float32), poisson=False)
    assert status == 2


def test_check_rules_and_tree():
    assert P.check_values(np.array([0.0, 1.0], np.float32), P.CHECK_FINITE_NONNEGATIVE) == 0
    assert P.check_values(np.array([-0.5], np.float32), P.CHECK_FINITE_NONNEGATIVE) == 1
    assert P.check_values(np.array([-0.5], np.float32), P.CHECK_FINITE) == 0
    assert P.check_values(np.array([np.inf], np.float32), P.CHECK_FINITE) == 1
    assert P.check_values(np.array([1.0], np.float32), P.CHECK_DECREMENT) == 1
    values = np.random.default_rng(5).normal(size=70000)
    assert P.tree_sum(values) == pytest.approx(math.fsum(values), rel=1e-12)
    assert P.tree_sum(np.zeros(0)) == 0.0
