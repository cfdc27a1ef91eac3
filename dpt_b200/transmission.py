"""Beer-Lambert transmission on CUDA: T = exp(-L), counts n0 T, log T = -L, removed 1 - T,
their VJPs and the inverse L = -log1p(-removed).

The interface follows the reference module (hcltech-robotics/dpt
``python/dpt/transmission.py``): ``TransmissionSpec`` declares the open-beam form and the
active inputs, ``prepare_transmission`` allocates the workspace (a status word and, for an
active shared beam, the FP64 reduction tree), and ``transmit`` / ``transmission_vjp`` /
``optical_depth_from_removed`` / ``optical_depth_from_removed_vjp`` write caller-owned
outputs.  Arrays are contiguous CUDA tensors, read flat; FP64 local arithmetic rounds once
into the FP32 destinations (``dpt_b200_transmit*`` in ``include/dpt_b200.h``).

Checked calls (``validate=True``) check the fixed inputs on the device before computing and
raise ``TransmissionError`` naming the first offending element, leaving every output
untouched; ``validate=False`` calls stay asynchronous and the caller accepts their results
with ``workspace.check_status()``.  Reverse-mode recording goes through the Torch operators
(``dpt_b200.torch.operators``), not a tape: ``tape`` must be None.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Literal

import torch

from . import _device as D
from . import _native as N
from .contracts import ContractError, NumericalError, binary32_scalar, integer, raise_device_status

BeamMode = Literal["none", "scalar", "device-scalar", "per-pixel"]
_BEAM_MODES = {"none": N.BEAM_NONE, "scalar": N.BEAM_SCALAR, "device-scalar": N.BEAM_DEVICE_SCALAR,
               "per-pixel": N.BEAM_PER_PIXEL}
_RULES = {"finite_nonnegative": N.CHECK_FINITE_NONNEGATIVE, "finite_seed": N.CHECK_FINITE,
          "decrement_domain": N.CHECK_DECREMENT}


class TransmissionError(ContractError):
    """Input, layout, aliasing or ownership violates the operator contract."""


class GradientRangeError(NumericalError):
    """A requested gradient cannot be represented in its binary32 destination."""


@dataclass(frozen=True, slots=True)
class TransmissionOutputs:
    """Selected caller-owned FP32 forward destinations (at least one)."""

    transmittance: torch.Tensor | None = None
    counts: torch.Tensor | None = None
    log_transmittance: torch.Tensor | None = None
    removed: torch.Tensor | None = None

    def __post_init__(self) -> None:
        if all(v is None for v in (self.transmittance, self.counts, self.log_transmittance, self.removed)):
            raise TransmissionError("request at least one output")


@dataclass(frozen=True, slots=True)
class TransmissionSpec:
    """Open-beam form (``none``, a host ``scalar``, a one-element ``device-scalar`` tensor or
    a ``per-pixel`` tensor) and the active inputs; the beam's value stays dynamic."""

    beam: BeamMode = "none"
    active_L: bool = True  # noqa: N815 - L is the optical depth throughout the API
    active_beam: bool = False

    def __post_init__(self) -> None:
        if self.beam not in _BEAM_MODES:
            raise TransmissionError(f"unsupported beam representation: {self.beam!r}")
        if type(self.active_L) is not bool or type(self.active_beam) is not bool:
            raise TransmissionError("active flags must be booleans")
        if self.active_beam and self.beam not in ("device-scalar", "per-pixel"):
            raise TransmissionError("an active beam must be a CUDA array, not a Python scalar")


class TransmissionWorkspace:
    """Status word and reduction scratch of one device; use it from one stream at a time.

    Inputs must stay unchanged until a backward pass that reads them completes."""

    def __init__(self, spec: TransmissionSpec, max_pixels: int, device: torch.device,
                 stream: torch.cuda.Stream | None) -> None:
        self.spec = spec
        self.max_pixels = max_pixels
        self.device = device
        self.stream = stream
        self.status = D.StatusWord(device)
        self._scratch = None
        if spec.active_beam and spec.beam == "device-scalar":
            self._scratch = D.reduction_scratch(max_pixels, device)

    @property
    def scratch_bytes(self) -> int:
        """Device scratch excluding caller-owned inputs, outputs and their adjoints."""
        return 4 + (0 if self._scratch is None else self._scratch.numel() * 8)

    def _stream(self, requested: torch.cuda.Stream | None = None) -> torch.cuda.Stream:
        return D.resolve_stream(self.stream, requested, self.device, TransmissionError)

    def clear_status(self) -> None:
        self.status.clear(self._stream())

    def check_status(self) -> None:
        """Synchronise the owning stream and reject any accumulated diagnostic (kept set)."""
        self._raise(self.status.read(self._stream()))

    def consume_status(self) -> None:
        """Deliver and reset one completed checkpoint, including reported errors."""
        self._raise(self.status.read(self._stream(), reset=True))

    def warm(self, **_ignored) -> tuple[str, ...]:
        """Kernels are compiled ahead of time: nothing to prepare."""
        return ()

    def _raise(self, code: int) -> None:
        raise_device_status(code, "transmission", {1: "invalid fixed device input",
                                                   2: "output or gradient cannot be represented"},
                            input_error=TransmissionError, range_error=GradientRangeError)


def prepare_transmission(spec: TransmissionSpec | None = None, *, device: str | torch.device = "cuda:0",
                         max_pixels: int, stream: torch.cuda.Stream | None = None) -> TransmissionWorkspace:
    """Allocate the status word (and an active shared beam's reduction tree), never outputs."""
    if spec is not None and not isinstance(spec, TransmissionSpec):
        raise TransmissionError("spec must be a TransmissionSpec")
    try:
        max_pixels = integer(max_pixels, "max_pixels")
    except ContractError as error:
        raise TransmissionError(str(error)) from error
    device = D.cuda_device(device, TransmissionError)
    N.library()
    return TransmissionWorkspace(spec or TransmissionSpec(), max_pixels, device, stream)


def _array(value, name: str, workspace: TransmissionWorkspace, count: int | None = None) -> int:
    return D.tensor(value, name, torch.float32, workspace.device, TransmissionError, count=count,
                    capacity=None if count == 1 else workspace.max_pixels)


def _beam(n0, count: int, workspace: TransmissionWorkspace) -> tuple[torch.Tensor | None, float]:
    mode = workspace.spec.beam
    if mode == "none":
        if n0 is not None:
            raise TransmissionError("this workspace declares no open-beam input")
        return None, 0.0
    if mode == "scalar":
        try:
            return None, binary32_scalar(n0, "n0", minimum=0.0)
        except ContractError as error:
            raise TransmissionError(str(error)) from error
    _array(n0, "n0", workspace, 1 if mode == "device-scalar" else count)
    return n0, 0.0


def _check_values(workspace: TransmissionWorkspace, stream: torch.cuda.Stream,
                  arrays: list[tuple[str, torch.Tensor | None, str]]) -> None:
    """Run the input rules on the device; on failure name the first offending element."""
    workspace._raise(workspace.status.read(stream))
    lib = N.library()
    for name, array, rule in arrays:
        if array is not None and array.numel():
            D.call(lib.dpt_b200_check_values(array.data_ptr(), array.numel(), _RULES[rule], workspace.status.ptr,
                                             stream.cuda_stream), f"check {name}")
    code = workspace.status.read(stream)
    if not code:
        return
    for name, array, rule in arrays:
        if array is None:
            continue
        values = array.reshape(-1).cpu()
        bad = ~torch.isfinite(values)
        if rule != "finite_seed":
            bad |= values < 0
        if rule == "decrement_domain":
            bad |= values >= 1
        found = torch.nonzero(bad)
        if found.numel():
            index = int(found[0, 0])
            raise TransmissionError(f"{name}[{index}]={float(values[index])!r} violates {rule}")
    workspace._raise(code)


def transmit(L: torch.Tensor, n0: float | torch.Tensor | None = None, *, out_T: torch.Tensor | None = None,
             out_counts: torch.Tensor | None = None, out_log_T: torch.Tensor | None = None,
             out_removed: torch.Tensor | None = None, outputs: TransmissionOutputs | None = None,
             workspace: TransmissionWorkspace, stream: torch.cuda.Stream | None = None, tape=None,
             validate: bool = True) -> None:
    """T = exp(-L), counts = n0 T, log_T = -L and removed = -expm1(-L).

    L is finite nonnegative FP32 optical depth (P pixels); each requested output is a
    caller-owned FP32 tensor of P elements.  n0 follows the workspace's beam form."""
    if tape is not None:
        raise TransmissionError("tape recording is not supported; use dpt_b200.torch.operators.transmit")
    if outputs is not None:
        if not isinstance(outputs, TransmissionOutputs):
            raise TransmissionError("outputs must be TransmissionOutputs")
        if any(v is not None for v in (out_T, out_counts, out_log_T, out_removed)):
            raise TransmissionError("supply outputs or individual transmission destinations")
        out_T, out_counts, out_log_T, out_removed = (outputs.transmittance, outputs.counts,
                                                     outputs.log_transmittance, outputs.removed)
    launch = workspace._stream(stream)
    count = _array(L, "L", workspace)
    beam, scalar = _beam(n0, count, workspace)
    destinations = (out_T, out_counts, out_log_T, out_removed)
    mask = sum(1 << i for i, v in enumerate(destinations) if v is not None)
    if mask == 0:
        raise TransmissionError("request at least one output")
    if out_counts is not None and workspace.spec.beam == "none":
        raise TransmissionError("counts require an explicit open-beam input")
    writes = []
    for name, value in zip(("out_T", "out_counts", "out_log_T", "out_removed"), destinations):
        if value is not None:
            _array(value, name, workspace, count)
            writes.append((name, value))
    D.disjoint([("L", L), ("n0", beam)], writes, TransmissionError)
    if validate:
        _check_values(workspace, launch, [("L", L, "finite_nonnegative"), ("n0", beam, "finite_nonnegative")])
    D.call(N.library().dpt_b200_transmit(L.data_ptr(), count, mask, _BEAM_MODES[workspace.spec.beam],
                                         D.ptr(beam), scalar, *(D.ptr(v) for v in destinations),
                                         launch.cuda_stream), "transmit")


def transmission_vjp(L: torch.Tensor, n0: float | torch.Tensor | None = None, *,
                     cotangent_T: torch.Tensor | None = None, cotangent_counts: torch.Tensor | None = None,
                     cotangent_log_T: torch.Tensor | None = None, cotangent_removed: torch.Tensor | None = None,
                     out_grad_L: torch.Tensor | None = None, out_grad_n0: torch.Tensor | None = None,
                     workspace: TransmissionWorkspace, stream: torch.cuda.Stream | None = None,
                     validate: bool = True, _accumulate: bool = False) -> None:
    """grad_L = -T cT - n0 T cCounts - cLog + T cRemoved; grad_n0 = T cCounts per pixel, or
    its fixed-order FP64 sum for a shared device-scalar beam.  Missing cotangents are zero;
    standalone calls overwrite their destinations."""
    launch = workspace._stream(stream)
    count = _array(L, "L", workspace)
    beam, scalar = _beam(n0, count, workspace)
    seeds = (cotangent_T, cotangent_counts, cotangent_log_T, cotangent_removed)
    if cotangent_counts is not None and workspace.spec.beam == "none":
        raise TransmissionError("a count cotangent requires an open-beam input")
    reads = [("L", L), ("n0", beam)]
    rules = [("L", L, "finite_nonnegative"), ("n0", beam, "finite_nonnegative")]
    for name, seed in zip(("cotangent_T", "cotangent_counts", "cotangent_log_T", "cotangent_removed"), seeds):
        if seed is not None:
            _array(seed, name, workspace, count)
            reads.append((name, seed))
            rules.append((name, seed, "finite_seed"))
    writes = []
    if out_grad_L is not None:
        if not workspace.spec.active_L:
            raise TransmissionError("L is declared fixed")
        _array(out_grad_L, "out_grad_L", workspace, count)
        writes.append(("out_grad_L", out_grad_L))
    if out_grad_n0 is not None:
        if not workspace.spec.active_beam:
            raise TransmissionError("n0 is declared fixed")
        _array(out_grad_n0, "out_grad_n0", workspace, 1 if workspace.spec.beam == "device-scalar" else count)
        writes.append(("out_grad_n0", out_grad_n0))
    if not writes:
        raise TransmissionError("request at least one active input gradient")
    D.disjoint(reads, writes, TransmissionError)
    if validate:
        _check_values(workspace, launch, rules)
    D.call(N.library().dpt_b200_transmit_vjp(
        L.data_ptr(), count, _BEAM_MODES[workspace.spec.beam], D.ptr(beam), scalar, *(D.ptr(s) for s in seeds),
        D.ptr(out_grad_L), D.ptr(out_grad_n0), D.ptr(workspace._scratch), int(_accumulate), workspace.status.ptr,
        launch.cuda_stream), "transmission_vjp")
    if validate:
        workspace.check_status()


def optical_depth_from_removed(delta: torch.Tensor, *, out_L: torch.Tensor, workspace: TransmissionWorkspace,
                               stream: torch.cuda.Stream | None = None, tape=None, validate: bool = True) -> None:
    """L = -log1p(-delta) inverts the removed fraction delta = 1 - T, 0 <= delta < 1."""
    if tape is not None:
        raise TransmissionError("tape recording is not supported")
    launch = workspace._stream(stream)
    count = _array(delta, "delta", workspace)
    _array(out_L, "out_L", workspace, count)
    D.disjoint([("delta", delta)], [("out_L", out_L)], TransmissionError)
    if validate:
        _check_values(workspace, launch, [("delta", delta, "decrement_domain")])
    D.call(N.library().dpt_b200_depth_from_removed(delta.data_ptr(), count, out_L.data_ptr(), launch.cuda_stream),
           "optical_depth_from_removed")


def optical_depth_from_removed_vjp(delta: torch.Tensor, cotangent: torch.Tensor, *, out_grad_delta: torch.Tensor,
                                   workspace: TransmissionWorkspace, stream: torch.cuda.Stream | None = None,
                                   validate: bool = True, _accumulate: bool = False) -> None:
    """grad_delta = cotangent / (1 - delta)."""
    launch = workspace._stream(stream)
    count = _array(delta, "delta", workspace)
    _array(cotangent, "cotangent", workspace, count)
    _array(out_grad_delta, "out_grad_delta", workspace, count)
    D.disjoint([("delta", delta), ("cotangent", cotangent)], [("out_grad_delta", out_grad_delta)],
               TransmissionError)
    if validate:
        _check_values(workspace, launch, [("delta", delta, "decrement_domain"),
                                          ("cotangent", cotangent, "finite_seed")])
    D.call(N.library().dpt_b200_depth_from_removed_vjp(delta.data_ptr(), cotangent.data_ptr(), count,
                                                       out_grad_delta.data_ptr(), int(_accumulate),
                                                       workspace.status.ptr, launch.cuda_stream),
           "optical_depth_from_removed_vjp")
    if validate:
        workspace.check_status()
