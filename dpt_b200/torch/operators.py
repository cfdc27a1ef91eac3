"""Transmission and scalar objectives as first-order Torch autograd operators.

Mirrors the reference adapter (hcltech-robotics/dpt ``python/dpt/torch/operators.py``):
``transmit`` returns an owned FP32 image (``T = exp(-L)``, counts ``n0 T``, ``-L`` or
``1 - T``) whose backward is the native transmission VJP, and ``objective`` returns an
owned FP64 scalar loss whose backward recomputes the image-space seed in FP64 and folds the
upstream scalar cotangent in before the single rounding to the prediction's dtype.
Observations, weights and masks are fixed.  Both operators run on the CUDA kernels of
``include/dpt_b200.h``; there is no CPU path.
"""

from __future__ import annotations

from typing import Literal

import torch

from ..contracts import ContractError, NumericalError
from ..objectives import ObjectiveWorkspace, evaluate_objective, objective_seed
from ..transmission import TransmissionWorkspace, transmission_vjp
from ..transmission import transmit as _transmit

TransmissionOutput = Literal["transmission", "counts", "log_transmission", "removed"]
__all__ = ["TransmissionOutput", "objective", "transmit"]
_OUTPUTS = {
    "transmission": ("out_T", "cotangent_T"),
    "counts": ("out_counts", "cotangent_counts"),
    "log_transmission": ("out_log_T", "cotangent_log_T"),
    "removed": ("out_removed", "cotangent_removed"),
}


def _tensor(value, name: str, dtype: torch.dtype) -> None:
    if not isinstance(value, torch.Tensor):
        raise ContractError(f"{name} must be a Torch tensor")
    if value.dtype != dtype or not value.is_contiguous():
        raise ContractError(f"{name} must use contiguous Torch {dtype} storage")


def _active(value: torch.Tensor, active: bool, name: str) -> None:
    if value.requires_grad and not active:
        raise ContractError(f"{name} was declared fixed in the native operator")


def _first_order() -> None:
    if torch.is_grad_enabled():
        raise ContractError("DPT Torch operators provide first-order derivatives only")


def _validate_flag(validate) -> None:
    if type(validate) is not bool:
        raise ContractError("validate must be a boolean")


class _Bridge:
    """Order a workspace's own stream after the caller's current stream and back again; a
    workspace without its own stream runs on the current stream directly."""

    def __init__(self, workspace, tensors) -> None:
        self.owned = workspace.stream
        self.tensors = [t for t in tensors if isinstance(t, torch.Tensor)]
        self.device = workspace.device

    def __enter__(self):
        self.current = torch.cuda.current_stream(self.device)
        if self.owned is not None and self.owned.cuda_stream != self.current.cuda_stream:
            self.owned.wait_stream(self.current)
            for tensor in self.tensors:
                tensor.record_stream(self.owned)
        return self

    def record(self, *tensors) -> None:
        if self.owned is not None and self.owned.cuda_stream != self.current.cuda_stream:
            for tensor in tensors:
                tensor.record_stream(self.owned)

    def __exit__(self, *exc) -> None:
        if self.owned is not None and self.owned.cuda_stream != self.current.cuda_stream:
            self.current.wait_stream(self.owned)


def _flat(value: torch.Tensor) -> torch.Tensor:
    return value.detach().reshape(-1)


class TransmissionFunction(torch.autograd.Function):
    @staticmethod
    def forward(owner, depth, beam, output: TransmissionOutput, workspace: TransmissionWorkspace, validate: bool):
        _validate_flag(validate)
        _tensor(depth, "optical_depth", torch.float32)
        _active(depth, workspace.spec.active_L, "optical_depth")
        if type(output) is not str or output not in _OUTPUTS:
            raise ContractError("select transmission, counts, log_transmission or removed")
        tensor_beam = isinstance(beam, torch.Tensor)
        if workspace.spec.beam in ("device-scalar", "per-pixel"):
            _tensor(beam, "open_beam", torch.float32)
            _active(beam, workspace.spec.active_beam, "open_beam")
            if beam.device != depth.device:
                raise ContractError("open_beam and optical_depth must share a device")
        elif tensor_beam:
            raise ContractError("Torch beam tensors require device-scalar or per-pixel policy")
        tensors = (depth, beam) if tensor_beam else (depth,)
        with _Bridge(workspace, tensors) as bridge:
            result = torch.empty_like(depth)
            bridge.record(result)
            _transmit(_flat(depth), _flat(beam) if tensor_beam else beam, **{_OUTPUTS[output][0]: _flat(result)},
                      workspace=workspace, stream=workspace.stream, validate=validate)
            workspace.consume_status()
        owner.save_for_backward(*tensors)
        owner.workspace, owner.output, owner.validate = workspace, output, validate
        owner.tensor_beam, owner.scalar_beam = tensor_beam, None if tensor_beam else beam
        return result

    @staticmethod
    def backward(owner, seed):
        _first_order()
        tensors = owner.saved_tensors
        depth = tensors[0]
        beam = tensors[1] if owner.tensor_beam else owner.scalar_beam
        workspace = owner.workspace
        with _Bridge(workspace, (*tensors, seed)) as bridge:
            seed = seed.to(torch.float32).contiguous()
            bridge.record(seed)
            grad_depth = torch.empty_like(depth) if owner.needs_input_grad[0] else None
            grad_beam = torch.empty_like(beam) if owner.tensor_beam and owner.needs_input_grad[1] else None
            bridge.record(*(v for v in (grad_depth, grad_beam) if v is not None))
            transmission_vjp(
                _flat(depth), _flat(beam) if owner.tensor_beam else beam,
                **{_OUTPUTS[owner.output][1]: _flat(seed)},
                out_grad_L=_flat(grad_depth) if grad_depth is not None else None,
                out_grad_n0=_flat(grad_beam) if grad_beam is not None else None,
                workspace=workspace, stream=workspace.stream, validate=owner.validate)
            workspace.consume_status()
        return grad_depth, grad_beam, None, None, None


class ObjectiveFunction(torch.autograd.Function):
    @staticmethod
    def forward(owner, prediction, observation, weights, valid, workspace: ObjectiveWorkspace, validate: bool):
        _validate_flag(validate)
        _tensor(prediction, "prediction", workspace.spec.dtype)
        _tensor(observation, "observation", torch.float32)
        fixed = [("observation", observation)]
        if weights is not None:
            _tensor(weights, "weights", torch.float32)
            fixed.append(("weights", weights))
        if valid is not None:
            _tensor(valid, "valid", torch.uint8)
            fixed.append(("valid", valid))
        for name, value in fixed:
            if value.requires_grad:
                raise ContractError(f"{name} is fixed in the native objective")
            if value.shape != prediction.shape:
                raise ContractError(f"{name} must have the prediction's shape")
        tensors = (prediction, *(value for _, value in fixed))
        with _Bridge(workspace, tensors) as bridge:
            result = torch.empty((), dtype=torch.float64, device=prediction.device)
            bridge.record(result)
            evaluate_objective(_flat(prediction), _flat(observation), out_loss=result.reshape(1),
                               weights=_flat(weights) if weights is not None else None,
                               valid=_flat(valid) if valid is not None else None,
                               workspace=workspace, stream=workspace.stream, validate=validate)
            workspace.consume_status()
        owner.save_for_backward(*tensors)
        owner.has_weights, owner.has_valid = weights is not None, valid is not None
        owner.workspace, owner.validate = workspace, validate
        return result

    @staticmethod
    def backward(owner, seed):
        _first_order()
        tensors = owner.saved_tensors
        prediction, observation = tensors[:2]
        weights = tensors[2] if owner.has_weights else None
        valid = tensors[-1] if owner.has_valid else None
        workspace = owner.workspace
        with _Bridge(workspace, (*tensors, seed)) as bridge:
            workspace.check_status()
            scale = float(seed.item())
            if scale != scale or scale in (float("inf"), float("-inf")):
                raise ContractError("objective cotangent must be finite")
            gradient = torch.zeros_like(prediction) if scale == 0 else torch.empty_like(prediction)
            bridge.record(gradient)
            if scale != 0:
                objective_seed(_flat(prediction), _flat(observation), scale=scale, out_cotangent=_flat(gradient),
                               weights=_flat(weights) if weights is not None else None,
                               valid=_flat(valid) if valid is not None else None,
                               workspace=workspace, stream=workspace.stream, validate=owner.validate)
                try:
                    workspace.consume_status()
                except NumericalError as error:
                    if type(error) is NumericalError:
                        raise NumericalError("Torch objective gradient exceeds its input storage range") from error
                    raise
        return gradient, None, None, None, None, None


def transmit(optical_depth: torch.Tensor, open_beam=None, *, output: TransmissionOutput = "transmission",
             workspace: TransmissionWorkspace, validate: bool = True) -> torch.Tensor:
    """``T = exp(-L)``, counts ``n0 T``, log transmission ``-L`` or removed ``1 - T``.

    ``optical_depth`` is nonnegative contiguous FP32 of any shape; the output keeps its
    shape.  ``workspace.spec.beam`` chooses no beam, a Python scalar, a one-element FP32
    tensor or a per-pixel FP32 tensor; ``active_L`` and ``active_beam`` select gradients."""
    return TransmissionFunction.apply(optical_depth, open_beam, output, workspace, validate)


def objective(prediction: torch.Tensor, observation: torch.Tensor, *, weights: torch.Tensor | None = None,
              valid: torch.Tensor | None = None, workspace: ObjectiveWorkspace,
              validate: bool = True) -> torch.Tensor:
    """Half squared error ``0.5 sum_p w_p (prediction_p - observation_p)^2`` or the Poisson
    half-deviance, as an owned FP64 scalar; only ``prediction`` has a gradient."""
    return ObjectiveFunction.apply(prediction, observation, weights, valid, workspace, validate)
