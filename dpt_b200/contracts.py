"""Error types and scalar argument checks shared by the projector's host code.

The error classes and the status-bit decoding follow the reference contracts
(hcltech-robotics/dpt ``python/dpt/contracts.py:15-119``): contract violations raise
``ContractError`` (a ``ValueError``), unrepresentable results raise
``NumericalError`` (a ``FloatingPointError``), and a field outside its physical
domain raises ``TrialDomainError``.
"""

from __future__ import annotations

import math
import struct
from numbers import Real
from typing import Any


class ContractError(ValueError):
    """A value, layout or ownership rule required by an operator was violated."""


class NumericalError(FloatingPointError):
    """An operation cannot represent its declared result; discard its outputs."""


class TrialDomainError(NumericalError):
    """A prediction or input lies outside its declared domain (status bit 8)."""


def integer(value: Any, name: str, *, minimum: int = 0, maximum: int = 2**31 - 1) -> int:
    """Require a Python ``int`` (not ``bool``) inside ``[minimum, maximum]``."""
    if type(value) is not int or not minimum <= value <= maximum:
        raise ContractError(f"{name} must be an integer in [{minimum}, {maximum}]")
    return value


def finite_scalar(value: Any, name: str, *, minimum: float | None = None) -> float:
    """Accept a finite real scalar with an optional inclusive lower bound."""
    if isinstance(value, bool) or not isinstance(value, Real):
        raise ContractError(f"{name} must be a real scalar")
    result = float(value)
    if not math.isfinite(result) or (minimum is not None and result < minimum):
        qualifier = "finite" if minimum is None else f"finite and at least {minimum}"
        raise ContractError(f"{name} must be {qualifier}")
    return result


def binary32_scalar(value: Any, name: str, *, minimum: float | None = None) -> float:
    """A finite real scalar rounded once to binary32; overflow to infinity is rejected."""
    result = finite_scalar(value, name, minimum=minimum)
    try:
        result = struct.unpack("f", struct.pack("f", result))[0]
    except (OverflowError, struct.error) as error:
        raise ContractError(f"{name} cannot be represented in binary32") from error
    if not math.isfinite(result):
        raise ContractError(f"{name} cannot be represented in binary32")
    return result


def finite_tuple(
    values: Any,
    name: str,
    *,
    positive: bool = False,
    minimum: float | None = 0.0,
    length: int | None = None,
) -> tuple[float, ...]:
    """Validate a non-empty tuple of finite scalars (non-negative unless minimum=None)."""
    if not isinstance(values, tuple) or not values:
        raise ContractError(f"{name} must be a non-empty immutable tuple")
    if length is not None and len(values) != length:
        raise ContractError(f"{name} must contain {length} values")
    result = tuple(finite_scalar(value, name, minimum=minimum) for value in values)
    if positive and any(value <= 0.0 for value in result):
        raise ContractError(f"{name} must be positive")
    return result


# Bit -> exception type, in precedence order (input errors first).
_STATUS_TYPES: tuple[tuple[int, type[Exception]], ...] = (
    (1, ContractError),
    (8, TrialDomainError),
    (2, NumericalError),
    (4, NumericalError),
)

PROJECTION_MESSAGES = {
    1: "invalid rigid pose coordinate map",
    2: "non-finite projection or gradient; discard these outputs",
    8: "field must be finite and non-negative",
    4: "numerical execution failure",
}


def raise_device_status(
    code: int,
    operator: str,
    messages: dict[int, str] | None = None,
    *,
    input_error: type[Exception] = ContractError,
    range_error: type[Exception] = NumericalError,
) -> None:
    """Raise the typed error for a nonzero device status word; do nothing for zero.

    Bit 1 raises ``input_error``, bit 8 ``TrialDomainError``, bit 2 ``range_error`` and
    bit 4 ``NumericalError``, in that precedence (reference ``contracts.py:90-119``)."""
    if not code:
        return
    descriptions = PROJECTION_MESSAGES if messages is None else messages
    for bit, error_type in _STATUS_TYPES:
        if code & bit:
            if bit == 1:
                error_type = input_error
            elif bit == 2:
                error_type = range_error
            raise error_type(f"{operator}: {descriptions.get(bit, 'device error')}")
    raise NumericalError(f"{operator}: unknown device status {code}")
