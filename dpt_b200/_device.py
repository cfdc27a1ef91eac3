"""Host-side plumbing shared by the image-space operators (transmission, objectives): the
status word and its pinned readback, tensor argument checks, overlap checks and the stream
a workspace enqueues on.

Workspaces follow the reference's ownership model (hcltech-robotics/dpt
``python/dpt/_runtime.py``): one workspace is used by one stream at a time, checked calls
synchronise that stream at their status checkpoints, and ``validate=False`` calls stay
asynchronous until the caller reads the status itself.
"""

from __future__ import annotations

import torch

from . import _native as N
from .contracts import ContractError

LIMIT = 2**31 - 1


def cuda_device(device: torch.device | str, error: type[Exception]) -> torch.device:
    device = torch.device(device)
    if device.type != "cuda":
        raise error("the B200 operators run on CUDA devices only")
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return device


class StatusWord:
    """One int32 device status word and its pinned host copy."""

    def __init__(self, device: torch.device) -> None:
        self.device = device
        self.word = torch.zeros(1, dtype=torch.int32, device=device)
        self.host = torch.zeros(1, dtype=torch.int32, pin_memory=True)

    @property
    def ptr(self) -> int:
        return self.word.data_ptr()

    def read(self, stream: torch.cuda.Stream, *, reset: bool = False) -> int:
        """Synchronise `stream` and return the word; with `reset`, clear it afterwards."""
        self.host.copy_(self.word, non_blocking=True)
        stream.synchronize()
        code = int(self.host[0])
        if reset and code:
            with torch.cuda.stream(stream):
                self.word.zero_()
        return code

    def clear(self, stream: torch.cuda.Stream) -> None:
        with torch.cuda.stream(stream):
            self.word.zero_()


def resolve_stream(owned: torch.cuda.Stream | None, requested: torch.cuda.Stream | None,
                   device: torch.device, error: type[Exception]) -> torch.cuda.Stream:
    """The stream a call enqueues on: the workspace's own stream when it has one (a different
    requested stream is an error), else the requested stream, else the current one."""
    if owned is not None:
        if requested is not None and requested.cuda_stream != owned.cuda_stream:
            raise error("this workspace is owned by another stream")
        return owned
    if requested is not None:
        return requested
    return torch.cuda.current_stream(device)


def tensor(value, name: str, dtype: torch.dtype, device: torch.device, error: type[Exception], *,
           count: int | None = None, capacity: int | None = None) -> int:
    """Check a contiguous device tensor of `dtype`; return its element count."""
    if not isinstance(value, torch.Tensor):
        raise error(f"{name} must be a Torch tensor")
    if value.dtype != dtype:
        raise error(f"{name} must have dtype {dtype}")
    if value.device != device:
        raise error(f"{name} must be on {device}")
    if not value.is_contiguous():
        raise error(f"{name} must be contiguous")
    size = value.numel()
    if count is not None and size != count:
        raise error(f"{name} must have {count} elements")
    if capacity is not None and size > capacity:
        raise error(f"{name} exceeds workspace capacity")
    if size > LIMIT:
        raise error(f"{name} has more than {LIMIT} elements")
    return size


def _span(value: torch.Tensor) -> tuple[int, int]:
    start = value.data_ptr()
    return start, start + value.numel() * value.element_size()


def disjoint(reads: list[tuple[str, torch.Tensor | None]], writes: list[tuple[str, torch.Tensor | None]],
             error: type[Exception]) -> None:
    """Reject a destination that overlaps an input or another destination."""
    reads = [(n, v) for n, v in reads if v is not None and v.numel()]
    writes = [(n, v) for n, v in writes if v is not None and v.numel()]
    for index, (name, value) in enumerate(writes):
        a0, a1 = _span(value)
        for other, tensor_ in reads + writes[index + 1:]:
            b0, b1 = _span(tensor_)
            if a0 < b1 and b0 < a1:
                raise error(f"{name} overlaps {other}")


def ptr(value: torch.Tensor | None) -> int | None:
    return None if value is None else value.data_ptr()


def call(code: int, what: str) -> None:
    N.check(code, what)


def reduction_scratch(count: int, device: torch.device) -> torch.Tensor:
    """FP64 scratch of the fixed reduction tree over `count` pixels."""
    nbytes = N.library().dpt_b200_reduction_bytes(count)
    if nbytes == 0:
        raise ContractError("reduction size out of range")
    return torch.empty(nbytes // 8, dtype=torch.float64, device=device)
