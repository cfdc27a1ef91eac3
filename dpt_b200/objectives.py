"""Image objectives on CUDA with an explicit measurement domain and image-space seed.

The interface follows the reference module (hcltech-robotics/dpt
``python/dpt/objectives.py``): ``ObjectiveSpec`` fixes the kind (half squared error or
Poisson half-deviance), the observation domain, the reduction (sum, or mean over the pixel
count), optional per-pixel weights and a uint8 validity mask, the prediction precision and
whether Poisson observations must be integers.  ``evaluate_objective`` writes the FP64 loss
and, optionally, the image-space seed d loss / d prediction in the prediction's dtype, in
one fused pass whose loss is reduced through a fixed FP64 tree (deterministic, no atomics;
``dpt_b200_objective`` in ``include/dpt_b200.h``).

Checked calls check the observation, weights, mask and prediction first and leave the
outputs untouched when they raise: ``ContractError`` for invalid fixed inputs,
``TrialDomainError`` for a Poisson prediction outside its domain, ``NumericalError`` for a
non-finite prediction or an unrepresentable result.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Literal

import torch

from . import _device as D
from . import _native as N
from .contracts import ContractError, integer, raise_device_status


@dataclass(frozen=True, slots=True)
class ObjectiveSpec:
    kind: Literal["squared_error", "poisson"] = "squared_error"
    domain: Literal["counts", "signal", "log_transmission"] = "signal"
    reduction: Literal["sum", "mean"] = "sum"
    weighted: bool = False
    masked: bool = False
    precision: Literal["float32", "float64"] = "float32"
    integer_counts: bool = True

    def __post_init__(self) -> None:
        if self.kind not in ("squared_error", "poisson"):
            raise ContractError("unsupported objective")
        if self.precision not in ("float32", "float64"):
            raise ContractError("objective precision must be float32 or float64")
        if self.domain not in ("counts", "signal", "log_transmission"):
            raise ContractError("declare the objective's measurement domain")
        if self.kind == "poisson" and self.domain != "counts":
            raise ContractError("a Poisson objective requires count-domain observations")
        if type(self.integer_counts) is not bool:
            raise ContractError("integer_counts must be a boolean")
        if self.reduction not in ("sum", "mean") or type(self.weighted) is not bool or type(self.masked) is not bool:
            raise ContractError("invalid objective reduction or weight policy")

    @property
    def dtype(self) -> torch.dtype:
        return torch.float64 if self.precision == "float64" else torch.float32

    @property
    def code(self) -> int:
        return N.OBJECTIVE_POISSON if self.kind == "poisson" else N.OBJECTIVE_SQUARED_ERROR


class ObjectiveWorkspace:
    """Status word and the loss reduction tree of one device; one stream at a time."""

    def __init__(self, spec: ObjectiveSpec, max_pixels: int, device: torch.device,
                 stream: torch.cuda.Stream | None) -> None:
        self.spec = spec
        self.max_pixels = max_pixels
        self.device = device
        self.stream = stream
        self.status = D.StatusWord(device)
        self._scratch = D.reduction_scratch(max_pixels, device)

    @property
    def scratch_bytes(self) -> int:
        return 4 + self._scratch.numel() * 8

    def _stream(self, requested: torch.cuda.Stream | None = None) -> torch.cuda.Stream:
        return D.resolve_stream(self.stream, requested, self.device, ContractError)

    def clear_status(self) -> None:
        self.status.clear(self._stream())

    def check_status(self) -> None:
        """Synchronise at an explicit acceptance boundary; failed outputs are unusable."""
        self._raise(self.status.read(self._stream()))

    def consume_status(self) -> None:
        """Deliver and reset one completed checkpoint, including reported errors."""
        self._raise(self.status.read(self._stream(), reset=True))

    def _raise(self, code: int) -> None:
        rule = "unmasked observations must be finite"
        if self.spec.kind == "poisson":
            rule += " and nonnegative"
            if self.spec.integer_counts:
                rule += " integer counts"
        if self.spec.weighted:
            rule += "; unmasked weights must be finite and nonnegative"
        if self.spec.masked:
            rule += "; validity masks must contain only 0 or 1"
        raise_device_status(code, "objectives", {1: rule, 2: "output or gradient cannot be represented",
                                                 8: "prediction outside trial domain",
                                                 4: "numerical execution failure"})

    def _inputs(self, size: int, weights, valid):
        if self.spec.weighted:
            D.tensor(weights, "weights", torch.float32, self.device, ContractError, count=size)
        elif weights is not None:
            raise ContractError("weights require a weighted objective specification")
        if self.spec.masked:
            D.tensor(valid, "valid", torch.uint8, self.device, ContractError, count=size)
        elif valid is not None:
            raise ContractError("valid requires a masked objective specification")

    def _check(self, stream, prediction, observation, weights, valid, size: int) -> None:
        self._raise(self.status.read(stream))
        if size:
            dtype = N.F64 if prediction is not None and prediction.dtype == torch.float64 else N.F32
            D.call(N.library().dpt_b200_objective_check(
                D.ptr(prediction), dtype, observation.data_ptr(), D.ptr(weights), D.ptr(valid), size,
                self.spec.code, int(self.spec.integer_counts), self.status.ptr, stream.cuda_stream),
                "objective check")
        self._raise(self.status.read(stream))

    def validate_observation(self, observation: torch.Tensor, *, weights: torch.Tensor | None = None,
                             valid: torch.Tensor | None = None, stream: torch.cuda.Stream | None = None) -> None:
        """Check fixed observations, weights and mask without a prediction."""
        launch = self._stream(stream)
        size = D.tensor(observation, "observation", torch.float32, self.device, ContractError)
        if size > self.max_pixels or (not size and self.spec.reduction == "mean"):
            raise ContractError("observation size is outside the objective capacity/domain")
        self._inputs(size, weights, valid)
        self._check(launch, None, observation, weights, valid, size)


def prepare_objective(spec: ObjectiveSpec, *, max_pixels: int, device: str | torch.device = "cuda:0",
                      stream: torch.cuda.Stream | None = None) -> ObjectiveWorkspace:
    """Allocate the status word and the FP64 reduction tree for up to `max_pixels` pixels."""
    if not isinstance(spec, ObjectiveSpec):
        raise ContractError("spec must be an ObjectiveSpec")
    capacity = integer(max_pixels, "max_pixels")
    device = D.cuda_device(device, ContractError)
    N.library()
    return ObjectiveWorkspace(spec, capacity, device, stream)


def _run(workspace: ObjectiveWorkspace, stream, prediction, observation, weights, valid, size: int, *,
         wide: bool, seed_scale: float, seed, loss) -> None:
    normalisation = 1.0 / size if workspace.spec.reduction == "mean" and size else 1.0
    dtype = N.F64 if prediction.dtype == torch.float64 else N.F32
    D.call(N.library().dpt_b200_objective(
        prediction.data_ptr(), dtype, int(wide), observation.data_ptr(), D.ptr(weights), D.ptr(valid), size,
        workspace.spec.code, normalisation, seed_scale, D.ptr(seed), workspace._scratch.data_ptr(), D.ptr(loss),
        workspace.status.ptr, stream.cuda_stream), "objective")


def evaluate_objective(prediction: torch.Tensor, observation: torch.Tensor, *, out_loss: torch.Tensor,
                       out_cotangent: torch.Tensor | None = None, weights: torch.Tensor | None = None,
                       valid: torch.Tensor | None = None, workspace: ObjectiveWorkspace,
                       stream: torch.cuda.Stream | None = None, validate: bool = True) -> None:
    """loss = sum_p valid_p w_p ell(prediction_p, observation_p) (divided by P for a mean).

    ell is 0.5 (mu - y)^2 or the Poisson half-deviance mu - y + y log(y / mu) (mu for
    y = 0).  prediction and out_cotangent have the spec's precision, observation and weights
    are FP32, valid is uint8 and out_loss is one FP64 element.  Masked pixels contribute zero
    loss and an exact zero seed."""
    spec = workspace.spec
    launch = workspace._stream(stream)
    size = D.tensor(prediction, "prediction", spec.dtype, workspace.device, ContractError)
    if size > workspace.max_pixels:
        raise ContractError("prediction exceeds workspace capacity")
    if size == 0 and spec.reduction == "mean":
        raise ContractError("a mean objective requires at least one pixel")
    D.tensor(observation, "observation", torch.float32, workspace.device, ContractError, count=size)
    D.tensor(out_loss, "out_loss", torch.float64, workspace.device, ContractError, count=1)
    workspace._inputs(size, weights, valid)
    if out_cotangent is not None:
        D.tensor(out_cotangent, "out_cotangent", spec.dtype, workspace.device, ContractError, count=size)
    D.disjoint([("prediction", prediction), ("observation", observation), ("weights", weights), ("valid", valid)],
               [("out_loss", out_loss), ("out_cotangent", out_cotangent)], ContractError)
    if validate:
        workspace._check(launch, prediction, observation, weights, valid, size)
    _run(workspace, launch, prediction, observation, weights, valid, size, wide=spec.precision == "float64",
         seed_scale=1.0, seed=out_cotangent, loss=out_loss)
    if validate:
        workspace.check_status()


def objective_seed(prediction: torch.Tensor, observation: torch.Tensor, *, scale: float,
                   out_cotangent: torch.Tensor, weights: torch.Tensor | None = None,
                   valid: torch.Tensor | None = None, workspace: ObjectiveWorkspace,
                   stream: torch.cuda.Stream | None = None, validate: bool = True) -> None:
    """The image-space seed alone, scaled by an upstream scalar cotangent before its single
    rounding: out = (w x d ell / d mu) x scale formed in FP64 (the FP64-precision forms for an
    FP32 prediction too), as the reference's Torch objective backward composes it
    (``python/dpt/torch/operators.py:322-354``).  Status bit 2 if a seed is not finite."""
    launch = workspace._stream(stream)
    size = D.tensor(prediction, "prediction", workspace.spec.dtype, workspace.device, ContractError,
                    capacity=workspace.max_pixels)
    D.tensor(observation, "observation", torch.float32, workspace.device, ContractError, count=size)
    D.tensor(out_cotangent, "out_cotangent", workspace.spec.dtype, workspace.device, ContractError, count=size)
    workspace._inputs(size, weights, valid)
    D.disjoint([("prediction", prediction), ("observation", observation), ("weights", weights), ("valid", valid)],
               [("out_cotangent", out_cotangent)], ContractError)
    if validate:
        workspace._check(launch, prediction, observation, weights, valid, size)
    _run(workspace, launch, prediction, observation, weights, valid, size, wide=True, seed_scale=float(scale),
         seed=out_cotangent, loss=None)


def reduce_objective_components(components: torch.Tensor, *, out_loss: torch.Tensor,
                                workspace: ObjectiveWorkspace, stream: torch.cuda.Stream | None = None,
                                validate: bool = True) -> None:
    """out_loss[0] = fixed-order FP64 sum of already weighted per-pixel terms (zero if empty)."""
    launch = workspace._stream(stream)
    if workspace.spec.reduction != "sum" or workspace.spec.weighted or workspace.spec.masked:
        raise ContractError("component reduction requires an unweighted sum workspace")
    size = D.tensor(components, "components", torch.float64, workspace.device, ContractError)
    if size > workspace.max_pixels:
        raise ContractError("components exceed reduction capacity")
    D.tensor(out_loss, "out_loss", torch.float64, workspace.device, ContractError, count=1)
    D.disjoint([("components", components)], [("out_loss", out_loss)], ContractError)
    if validate:
        workspace.check_status()
    D.call(N.library().dpt_b200_reduce_sum(components.data_ptr(), size, workspace._scratch.data_ptr(),
                                           out_loss.data_ptr(), workspace.status.ptr, launch.cuda_stream),
           "reduce_objective_components")
    if validate:
        workspace.check_status()
