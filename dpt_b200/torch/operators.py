"""Transmission and scalar objectives as first-order Torch autograd operators.

Same operators as the reference adapter (hcltech-robotics/dpt ``python/dpt/torch/operators.py``):
``transmit`` returns an owned FP32 image (``T = exp(-L)``, counts ``n0 T``, ``-L`` or
``1 - T``) whose backward is the native transmission VJP, and ``objective`` returns an owned
FP64 scalar loss whose backward recomputes the image-space seed in FP64 with the upstream
scalar cotangent folded in before the single rounding to the prediction's dtype.
Observations, weights and masks are fixed.  Both run on the CUDA kernels of
``include/dpt_b200.h``; there is no CPU path.

Argument rules (``ContractError`` with the message shown, checked top to bottom):

==================  ==========================================================================
both operators      ``validate`` a bool -- "validate must be a boolean"; a tensor operand
                    -- "<name> must be a Torch tensor", of contiguous storage of its dtype --
                    "<name> must use contiguous Torch <dtype> storage"; backward under
                    grad mode -- "DPT Torch operators provide first-order derivatives only"
``transmit``        ``optical_depth`` FP32, differentiable only when the workspace declares
                    it active -- "optical_depth was declared fixed in the native operator";
                    ``output`` one of the four names -- "select transmission, counts,
                    log_transmission or removed"; a tensor ``open_beam`` only for the
                    device-scalar and per-pixel beam policies -- "Torch beam tensors require
                    device-scalar or per-pixel policy", then FP32, active rule as above, on
                    the depth's device -- "open_beam and optical_depth must share a device"
``objective``       ``prediction`` of the workspace dtype; ``observation`` FP32, ``weights``
                    FP32, ``valid`` uint8 (each optional operand type-checked in that order),
                    then each fixed operand in that order: no gradient -- "<name> is fixed in
                    the native objective", the prediction's shape -- "<name> must have the
                    prediction's shape"; backward: a finite upstream cotangent -- "objective
                    cotangent must be finite"; a gradient beyond the prediction's range raises
                    NumericalError "Torch objective gradient exceeds its input storage range"
==================  ==========================================================================
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Literal

import torch

from ..contracts import ContractError, NumericalError
from ..objectives import ObjectiveWorkspace, evaluate_objective, objective_seed
from ..transmission import TransmissionWorkspace, transmission_vjp
from ..transmission import transmit as _transmit

TransmissionOutput = Literal["transmission", "counts", "log_transmission", "removed"]
__all__ = ["TransmissionOutput", "objective", "transmit"]

# output name -> (keyword of its forward buffer, keyword of its cotangent in the VJP)
_KEYWORDS = {
    "transmission": ("out_T", "cotangent_T"),
    "counts": ("out_counts", "cotangent_counts"),
    "log_transmission": ("out_log_T", "cotangent_log_T"),
    "removed": ("out_removed", "cotangent_removed"),
}
_TENSOR_BEAMS = ("device-scalar", "per-pixel")


def _require_tensor(value, name: str, dtype: torch.dtype) -> torch.Tensor:
    if not isinstance(value, torch.Tensor):
        raise ContractError(f"{name} must be a Torch tensor")
    if value.dtype != dtype or not value.is_contiguous():
        raise ContractError(f"{name} must use contiguous Torch {dtype} storage")
    return value


def _require_bool(validate) -> bool:
    if type(validate) is not bool:
        raise ContractError("validate must be a boolean")
    return validate


def _require_first_order() -> None:
    if torch.is_grad_enabled():
        raise ContractError("DPT Torch operators provide first-order derivatives only")


def _vector(value: torch.Tensor | None) -> torch.Tensor | None:
    return None if value is None else value.detach().reshape(-1)


class _OnWorkspaceStream:
    """Run native work on the workspace's own stream (when it has one) ordered after the
    caller's current stream, and order the caller's stream after it on exit; tensors used on
    that stream are recorded there so the caching allocator keeps them alive."""

    def __init__(self, workspace, tensors) -> None:
        self.stream = workspace.stream
        self.device = workspace.device
        self.tensors = [value for value in tensors if isinstance(value, torch.Tensor)]

    def __enter__(self) -> _OnWorkspaceStream:
        self.caller = torch.cuda.current_stream(self.device)
        self.separate = self.stream is not None and self.stream.cuda_stream != self.caller.cuda_stream
        if self.separate:
            self.stream.wait_stream(self.caller)
        self.keep(*self.tensors)
        return self

    def keep(self, *tensors) -> None:
        if self.separate:
            for value in tensors:
                value.record_stream(self.stream)

    def __exit__(self, *exc) -> None:
        if self.separate:
            self.caller.wait_stream(self.stream)


@dataclass
class _TransmissionCall:
    """One ``transmit`` call: its workspace, output, checking policy and beam form."""

    workspace: TransmissionWorkspace
    output: str
    validate: bool
    beam_is_tensor: bool
    scalar_beam: object = None

    @classmethod
    def checked(cls, depth, beam, output, workspace: TransmissionWorkspace, validate) -> _TransmissionCall:
        validate = _require_bool(validate)
        spec = workspace.spec
        _require_tensor(depth, "optical_depth", torch.float32)
        if depth.requires_grad and not spec.active_L:
            raise ContractError("optical_depth was declared fixed in the native operator")
        if type(output) is not str or output not in _KEYWORDS:
            raise ContractError("select transmission, counts, log_transmission or removed")
        beam_is_tensor = isinstance(beam, torch.Tensor)
        if spec.beam in _TENSOR_BEAMS:
            _require_tensor(beam, "open_beam", torch.float32)
            if beam.requires_grad and not spec.active_beam:
                raise ContractError("open_beam was declared fixed in the native operator")
            if beam.device != depth.device:
                raise ContractError("open_beam and optical_depth must share a device")
        elif beam_is_tensor:
            raise ContractError("Torch beam tensors require device-scalar or per-pixel policy")
        return cls(workspace, output, validate, beam_is_tensor, None if beam_is_tensor else beam)

    def native_beam(self, beam):
        return _vector(beam) if self.beam_is_tensor else self.scalar_beam

    def forward(self, depth: torch.Tensor, beam) -> torch.Tensor:
        inputs = (depth, beam) if self.beam_is_tensor else (depth,)
        with _OnWorkspaceStream(self.workspace, inputs) as scope:
            result = torch.empty_like(depth)
            scope.keep(result)
            _transmit(_vector(depth), self.native_beam(beam), **{_KEYWORDS[self.output][0]: _vector(result)},
                      workspace=self.workspace, stream=self.workspace.stream, validate=self.validate)
            self.workspace.consume_status()
        return result

    def backward(self, depth: torch.Tensor, beam, seed: torch.Tensor, wants: tuple[bool, bool]):
        with _OnWorkspaceStream(self.workspace, (depth, beam, seed)) as scope:
            seed = seed.to(torch.float32).contiguous()
            scope.keep(seed)
            grad_depth = torch.empty_like(depth) if wants[0] else None
            grad_beam = torch.empty_like(beam) if self.beam_is_tensor and wants[1] else None
            scope.keep(*(g for g in (grad_depth, grad_beam) if g is not None))
            transmission_vjp(_vector(depth), self.native_beam(beam), **{_KEYWORDS[self.output][1]: _vector(seed)},
                             out_grad_L=_vector(grad_depth), out_grad_n0=_vector(grad_beam),
                             workspace=self.workspace, stream=self.workspace.stream, validate=self.validate)
            self.workspace.consume_status()
        return grad_depth, grad_beam


class TransmissionFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, depth, beam, output: TransmissionOutput, workspace: TransmissionWorkspace, validate: bool):
        call = _TransmissionCall.checked(depth, beam, output, workspace, validate)
        result = call.forward(depth, beam)
        ctx.call = call
        ctx.save_for_backward(depth, beam if call.beam_is_tensor else None)
        return result

    @staticmethod
    def backward(ctx, seed):
        _require_first_order()
        depth, beam = ctx.saved_tensors
        call: _TransmissionCall = ctx.call
        grad_depth, grad_beam = call.backward(depth, beam if call.beam_is_tensor else None, seed,
                                              (ctx.needs_input_grad[0], ctx.needs_input_grad[1]))
        return grad_depth, grad_beam, None, None, None


@dataclass
class _ObjectiveCall:
    """One ``objective`` call: its workspace, checking policy and which optional operands exist."""

    workspace: ObjectiveWorkspace
    validate: bool

    @classmethod
    def checked(cls, prediction, observation, weights, valid, workspace: ObjectiveWorkspace,
                validate) -> _ObjectiveCall:
        validate = _require_bool(validate)
        _require_tensor(prediction, "prediction", workspace.spec.dtype)
        fixed = {"observation": _require_tensor(observation, "observation", torch.float32)}
        if weights is not None:
            fixed["weights"] = _require_tensor(weights, "weights", torch.float32)
        if valid is not None:
            fixed["valid"] = _require_tensor(valid, "valid", torch.uint8)
        for name, value in fixed.items():
            if value.requires_grad:
                raise ContractError(f"{name} is fixed in the native objective")
            if value.shape != prediction.shape:
                raise ContractError(f"{name} must have the prediction's shape")
        return cls(workspace, validate)

    def loss(self, prediction, observation, weights, valid) -> torch.Tensor:
        with _OnWorkspaceStream(self.workspace, (prediction, observation, weights, valid)) as scope:
            result = torch.empty((), dtype=torch.float64, device=prediction.device)
            scope.keep(result)
            evaluate_objective(_vector(prediction), _vector(observation), out_loss=result.reshape(1),
                               weights=_vector(weights), valid=_vector(valid), workspace=self.workspace,
                               stream=self.workspace.stream, validate=self.validate)
            self.workspace.consume_status()
        return result

    def gradient(self, prediction, observation, weights, valid, seed: torch.Tensor) -> torch.Tensor:
        with _OnWorkspaceStream(self.workspace, (prediction, observation, weights, valid, seed)) as scope:
            self.workspace.check_status()
            scale = float(seed.item())
            if scale - scale != 0.0:  # NaN or infinite
                raise ContractError("objective cotangent must be finite")
            if scale == 0.0:
                gradient = torch.zeros_like(prediction)
                scope.keep(gradient)
                return gradient
            gradient = torch.empty_like(prediction)
            scope.keep(gradient)
            objective_seed(_vector(prediction), _vector(observation), scale=scale, out_cotangent=_vector(gradient),
                           weights=_vector(weights), valid=_vector(valid), workspace=self.workspace,
                           stream=self.workspace.stream, validate=self.validate)
            try:
                self.workspace.consume_status()
            except NumericalError as error:
                # a plain range failure means the FP64 seed overflowed the prediction's dtype;
                # typed subclasses (an input outside its domain) pass through
                if type(error) is not NumericalError:
                    raise
                raise NumericalError("Torch objective gradient exceeds its input storage range") from error
        return gradient


class ObjectiveFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, prediction, observation, weights, valid, workspace: ObjectiveWorkspace, validate: bool):
        call = _ObjectiveCall.checked(prediction, observation, weights, valid, workspace, validate)
        result = call.loss(prediction, observation, weights, valid)
        ctx.call = call
        ctx.save_for_backward(prediction, observation, weights, valid)
        return result

    @staticmethod
    def backward(ctx, seed):
        _require_first_order()
        prediction, observation, weights, valid = ctx.saved_tensors
        gradient = ctx.call.gradient(prediction, observation, weights, valid, seed)
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
