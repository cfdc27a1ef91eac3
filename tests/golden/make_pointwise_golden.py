"""Generate ``pointwise.npz``: golden vectors of the transmission and objective operators from
the reference project's own exact-input Decimal oracles.  Run with the reference checkout
given by ``--reference PATH`` or ``DPT_REFERENCE`` (these modules import without Warp):

    python tests/golden/make_pointwise_golden.py --reference PATH

Sources used (paths inside the reference project):
  * python/dpt/validation/transmission.py - forward_reference, inverse_reference,
    vjp_reference, inverse_vjp_reference, scalar_beam_reference, round_binary32
    (100-digit Decimal evaluation at the exact binary32 inputs)
  * python/dpt/validation/objectives.py - scalar_objective (100-digit Decimal)
The inputs (binade edges and their neighbours, the cancellation seams of the removed
fraction and of the Poisson half-deviance, seeded random values) are generated here.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from reference_checkout import reference_root  # noqa: E402

REFERENCE = reference_root()

from dpt.validation import objectives as ro  # noqa: E402
from dpt.validation import transmission as rt  # noqa: E402

F32_MAX = float(np.finfo(np.float32).max)


def small_points() -> np.ndarray:
    """Binade edges 2^-149 .. 2^-1 with their float32 neighbours, the seams 2^-25, 1/8, 1/2, 1
    with neighbours, signed zeros and seeded values in [0, 1)."""
    edges = np.array([2.0**e for e in range(-149, 0)], dtype=np.float32)
    seams = np.array([2.0**-25, 0.125, 0.5, 1.0], dtype=np.float32)
    rng = np.random.default_rng(20240611)
    values = np.concatenate([
        np.nextafter(edges, np.float32(0)), edges, np.nextafter(edges, np.float32(1)),
        np.nextafter(seams, np.float32(0)), seams[:-1], np.nextafter(seams[:-1], np.float32(1)),
        np.array([0.0, -0.0], dtype=np.float32),
        rng.integers(0, 0x3F800000, 384, dtype=np.uint32).view(np.float32),
        rng.uniform(0, 1, 768).astype(np.float32),
    ])
    return values.astype(np.float32)


def forward_cases():
    depth = np.concatenate([
        small_points(),
        np.array([1.0, 2.0, 10.0, 63.99, 64.0, 64.01, 87.0, 103.0, 104.0, 110.0, 200.0, 745.0, 1024.0, F32_MAX],
                 dtype=np.float32),
        np.random.default_rng(7).uniform(0, 90, 256).astype(np.float32),
    ])
    beams = np.array([1.0, 1.0e30, 2.0**-149, 1000.0, 0.0, 3.5, F32_MAX], dtype=np.float32)
    beam = beams[np.arange(depth.size) % beams.size]
    rows = [rt.forward_reference(float(x), float(n), precision=100).rounded() for x, n in zip(depth, beam)]
    return {
        "forward_depth": depth,
        "forward_beam": beam,
        "forward_T": np.array([r["T"] for r in rows], dtype=np.float32),
        "forward_counts": np.array([r["counts"] for r in rows], dtype=np.float32),
        "forward_log_T": np.array([r["log_T"] for r in rows], dtype=np.float32),
        "forward_removed": np.array([r["removed"] for r in rows], dtype=np.float32),
    }


def inverse_cases():
    delta = small_points()
    delta = np.concatenate([delta[delta < 1], np.array([1 - 2.0**-24, 0.75, 0.999], dtype=np.float32)])
    depth = np.array([rt.round_binary32(rt.inverse_reference(float(x), precision=100)) for x in delta],
                     dtype=np.float32)
    rng = np.random.default_rng(11)
    seed = rng.uniform(-4, 4, delta.size).astype(np.float32)
    grads = [rt.inverse_vjp_reference(float(x), float(s)) for x, s in zip(delta, seed)]
    return {
        "inverse_delta": delta,
        "inverse_depth": depth,
        "inverse_seed": seed,
        "inverse_grad": np.array([float(g) for g, _ in grads]),
        "inverse_budget": np.array([float(b) for _, b in grads]),
    }


def vjp_cases():
    rng = np.random.default_rng(23)
    n = 640
    depth = np.concatenate([rng.uniform(0, 12, n - 8),
                            np.array([0.0, 2.0**-149, 64.0, 70.0, 110.0, 200.0, 1024.0, 0.5])]).astype(np.float32)
    beam = rng.uniform(0, 2000, n).astype(np.float32)
    seeds = {name: rng.uniform(-3, 3, n).astype(np.float32) for name in ("T", "counts", "log_T", "removed")}
    rows = [rt.vjp_reference(float(depth[i]), float(beam[i]), seed_T=float(seeds["T"][i]),
                             seed_counts=float(seeds["counts"][i]), seed_log_T=float(seeds["log_T"][i]),
                             seed_removed=float(seeds["removed"][i])) for i in range(n)]
    # the shared-beam sum in the kernels' order: 640 pixels fall in one 2048-pixel block, whose
    # threads add their (up to) 8 terms in sequence before a depth-8 pairwise tree over the
    # 256 threads, so the longest path has 16 additions
    total, budget = rt.scalar_beam_reference(depth.tolist(), seeds["counts"].tolist(), addition_depth=16)
    return {
        "vjp_depth": depth,
        "vjp_beam": beam,
        **{f"vjp_seed_{k}": v for k, v in seeds.items()},
        "vjp_grad_L": np.array([float(r.grad_L) for r in rows]),
        "vjp_budget_L": np.array([float(r.budget_L) for r in rows]),
        "vjp_grad_n0": np.array([float(r.grad_n0) for r in rows]),
        "vjp_budget_n0": np.array([float(r.budget_n0) for r in rows]),
        "vjp_shared_n0": np.array([float(total)]),
        "vjp_shared_budget": np.array([float(budget)]),
    }


def objective_cases():
    ratios = [np.nextafter(0.001, 0.0), 0.001, np.nextafter(0.001, 1.0), 0.0010001, np.nextafter(0.25, 0.0), 0.25,
              np.nextafter(0.25, 1.0), *np.geomspace(1e-9, 0.99, 48).tolist()]
    predicted, observed = [], []
    for y in (1.0, float(2**20), float(np.float32(1e20))):
        for r in ratios:
            for sign in (-1.0, 1.0):
                predicted.append(y * (1.0 + sign * r))
                observed.append(y)
    # far from equality, a zero observation and small/large predictions
    for mu, y in ((3.0, 0.0), (0.0, 0.0), (1e-300, 5.0), (1e300, 7.0), (50.0, 3.0), (0.02, 9.0)):
        predicted.append(mu)
        observed.append(y)
    poisson = [ro.scalar_objective(p, y, poisson=True) for p, y in zip(predicted, observed)]
    rng = np.random.default_rng(31)
    sq_pred = rng.normal(0, 100, 256)
    sq_obs = rng.normal(0, 100, 256).astype(np.float32).astype(np.float64)
    squared = [ro.scalar_objective(float(p), float(y), poisson=False) for p, y in zip(sq_pred, sq_obs)]
    # the 117-pixel repeating Poisson pattern (prediction 1 + i % 13, observation i % 9)
    pattern = [ro.scalar_objective(float(1 + i % 13), float(i % 9), poisson=True) for i in range(117)]
    return {
        "poisson_prediction": np.array(predicted),
        "poisson_observation": np.array(observed),
        "poisson_loss": np.array([float(v) for v, _ in poisson]),
        "poisson_derivative": np.array([float(d) for _, d in poisson]),
        "squared_prediction": sq_pred,
        "squared_observation": sq_obs,
        "squared_loss": np.array([float(v) for v, _ in squared]),
        "squared_derivative": np.array([float(d) for _, d in squared]),
        "pattern_loss": np.array([float(v) for v, _ in pattern]),
        "pattern_derivative": np.array([float(d) for _, d in pattern]),
    }


def main() -> None:
    arrays = {**forward_cases(), **inverse_cases(), **vjp_cases(), **objective_cases()}
    np.savez_compressed(HERE / "pointwise.npz", **arrays)
    print({k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
