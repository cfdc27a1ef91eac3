"""ctypes wrapper of the CPU pointwise oracle (``pointwise_oracle.c``).  TEST INFRASTRUCTURE
ONLY: the checker of the CUDA transmission and objective kernels, never the product.

Arguments and results are numpy arrays; a ``None`` cotangent is zero, a ``None`` weight or
mask is absent.  Every function returns its outputs and the status bits it would set.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import build as _build

BEAM_NONE, BEAM_SCALAR, BEAM_DEVICE_SCALAR, BEAM_PER_PIXEL = 0, 1, 2, 3
CHECK_FINITE_NONNEGATIVE, CHECK_FINITE, CHECK_DECREMENT = 0, 1, 2

_lib = None


def library():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(_build.build()))
        V, L, I, F, D = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float, ctypes.c_double
        signatures = {
            "oracle_tree_sum": ([V, L], D),
            "oracle_poisson_half_deviance": ([D, D], D),
            "oracle_check_values": ([V, L, I], I),
            "oracle_transmit": ([V, L, I, V, F, V, V, V, V], None),
            "oracle_transmit_vjp": ([V, L, I, V, F, V, V, V, V, V, V, V], I),
            "oracle_depth_from_removed": ([V, L, V], None),
            "oracle_depth_from_removed_vjp": ([V, V, L, V], I),
            "oracle_objective_check": ([V, I, V, V, V, L, I, I], I),
            "oracle_objective": ([V, I, I, V, V, V, L, I, D, D, V, V], I),
        }
        for name, (argtypes, restype) in signatures.items():
            function = getattr(lib, name)
            function.argtypes = argtypes
            function.restype = restype
        _lib = lib
    return _lib


def _f32(values) -> np.ndarray | None:
    return None if values is None else np.ascontiguousarray(values, dtype=np.float32).reshape(-1)


def _ptr(array: np.ndarray | None) -> int | None:
    return None if array is None else array.ctypes.data


def check_values(values, rule: int) -> int:
    values = _f32(values)
    return library().oracle_check_values(_ptr(values), values.size, rule)


def transmit(depth, *, beam_mode: int = BEAM_NONE, beam=None, beam_scalar: float = 0.0):
    """Return (transmission, counts or None, log_transmission, removed)."""
    depth = _f32(depth)
    beam = _f32(beam)
    n = depth.size
    t, log_t, removed = (np.empty(n, np.float32) for _ in range(3))
    counts = np.empty(n, np.float32) if beam_mode != BEAM_NONE else None
    library().oracle_transmit(_ptr(depth), n, beam_mode, _ptr(beam), beam_scalar, _ptr(t), _ptr(counts),
                              _ptr(log_t), _ptr(removed))
    return t, counts, log_t, removed


def transmit_vjp(depth, *, beam_mode: int = BEAM_NONE, beam=None, beam_scalar: float = 0.0,
                 seed_transmission=None, seed_counts=None, seed_log=None, seed_removed=None,
                 beam_gradient: str | None = None):
    """Return (grad_depth, grad_beam or None, status); ``beam_gradient`` is None,
    "per-pixel" or "shared"."""
    depth = _f32(depth)
    beam = _f32(beam)
    seeds = [_f32(s) for s in (seed_transmission, seed_counts, seed_log, seed_removed)]
    n = depth.size
    grad = np.empty(n, np.float32)
    pixels = np.empty(n, np.float32) if beam_gradient == "per-pixel" else None
    shared = np.empty(1, np.float32) if beam_gradient == "shared" else None
    status = library().oracle_transmit_vjp(_ptr(depth), n, beam_mode, _ptr(beam), beam_scalar,
                                           *(_ptr(s) for s in seeds), _ptr(grad), _ptr(pixels), _ptr(shared))
    return grad, pixels if pixels is not None else shared, status


def depth_from_removed(removed) -> np.ndarray:
    removed = _f32(removed)
    depth = np.empty(removed.size, np.float32)
    library().oracle_depth_from_removed(_ptr(removed), removed.size, _ptr(depth))
    return depth


def depth_from_removed_vjp(removed, seed):
    removed, seed = _f32(removed), _f32(seed)
    grad = np.empty(removed.size, np.float32)
    status = library().oracle_depth_from_removed_vjp(_ptr(removed), _ptr(seed), removed.size, _ptr(grad))
    return grad, status


def _prediction(prediction):
    prediction = np.ascontiguousarray(prediction).reshape(-1)
    if prediction.dtype not in (np.float32, np.float64):
        prediction = prediction.astype(np.float32)
    return prediction, int(prediction.dtype == np.float64)


def objective_check(prediction, observation, *, weights=None, valid=None, poisson: bool,
                    integer_counts: bool = True) -> int:
    observation = _f32(observation)
    if prediction is not None:
        prediction, dtype = _prediction(prediction)
    else:
        dtype = 0
    valid = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint8).reshape(-1)
    return library().oracle_objective_check(_ptr(prediction), dtype, _ptr(observation), _ptr(_f32(weights)),
                                            _ptr(valid), observation.size, int(poisson), int(integer_counts))


def objective(prediction, observation, *, weights=None, valid=None, poisson: bool, wide: bool | None = None,
              normalisation: float = 1.0, seed_scale: float = 1.0):
    """Return (loss, seed in the prediction's dtype, status)."""
    prediction, dtype = _prediction(prediction)
    observation = _f32(observation)
    weights = _f32(weights)
    valid = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint8).reshape(-1)
    seed = np.empty(prediction.size, prediction.dtype)
    loss = np.empty(1, np.float64)
    wide = bool(dtype) if wide is None else wide
    status = library().oracle_objective(_ptr(prediction), dtype, int(wide), _ptr(observation), _ptr(weights),
                                        _ptr(valid), prediction.size, int(poisson), normalisation, seed_scale,
                                        _ptr(seed), _ptr(loss))
    return float(loss[0]), seed, status


def tree_sum(values) -> float:
    values = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    return library().oracle_tree_sum(_ptr(values), values.size)


def poisson_half_deviance(predicted: float, observed: float) -> float:
    return library().oracle_poisson_half_deviance(predicted, observed)
