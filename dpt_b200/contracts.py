"""Error types and scalar argument checks shared by the projector's host code.

The error classes and the status-bit decoding follow the reference contracts
(hcltech-robotics/dpt ``python/dpt/contracts.py:15-119``): contract violations raise
``ContractError`` (a ``ValueError``), unrepresentable results raise
``NumericalError`` (a ``FloatingPointError``), and a field outside its physical
domain raises ``TrialDomainError``.
"""

from __future__ import annotations

import math
from array import array
from numbers import Real
from typing import Any


class ContractError(ValueError):
    """A value, layout or ownership rule required by an operator was violated."""


class NumericalError(FloatingPointError):
    """An operation cannot represent its declared result; discard its outputs."""


class TrialDomainError(NumericalError):
    """A prediction or input lies outside its declared domain (status bit 8)."""


def _plain_real(value: Any) -> bool:
    return isinstance(value, Real) and not isinstance(value, bool)


def integer(value: Any, name: str, *, minimum: int = 0, maximum: int = 2**31 - 1) -> int:
    """A Python ``int`` (``bool`` and other subclasses excluded) in ``[minimum, maximum]``."""
    if type(value) is not int or value < minimum or value > maximum:
        raise ContractError(f"{name} must be an integer in [{minimum}, {maximum}]")
    return value


def finite_scalar(value: Any, name: str, *, minimum: float | None = None) -> float:
    """A real scalar (``bool`` excluded) as a finite Python float, at least ``minimum``."""
    if not _plain_real(value):
        raise ContractError(f"{name} must be a real scalar")
    number = float(value)
    if minimum is None:
        if not math.isfinite(number):
            raise ContractError(f"{name} must be finite")
    elif not (math.isfinite(number) and number >= minimum):
        raise ContractError(f"{name} must be finite and at least {minimum}")
    return number


# Finite doubles at or above this magnitude round to infinity in binary32 (round to nearest:
# halfway between the largest binary32 value and 2^128).
_BINARY32_OVERFLOW = 2.0**128 - 2.0**103


def binary32_scalar(value: Any, name: str, *, minimum: float | None = None) -> float:
    """A finite real scalar rounded once to binary32; a value that rounds to infinity is rejected."""
    number = finite_scalar(value, name, minimum=minimum)
    if abs(number) >= _BINARY32_OVERFLOW:
        raise ContractError(f"{name} cannot be represented in binary32")
    return float(array("f", (number,))[0])


def finite_tuple(
    values: Any,
    name: str,
    *,
    positive: bool = False,
    minimum: float | None = 0.0,
    length: int | None = None,
) -> tuple[float, ...]:
    """A non-empty tuple of finite scalars (each at least ``minimum`` unless it is None), of
    ``length`` entries when given, all strictly positive when ``positive``."""
    if not (isinstance(values, tuple) and len(values) > 0):
        raise ContractError(f"{name} must be a non-empty immutable tuple")
    if length is not None and len(values) != length:
        raise ContractError(f"{name} must contain {length} values")
    numbers = [finite_scalar(entry, name, minimum=minimum) for entry in values]
    if positive and min(numbers) <= 0.0:
        raise ContractError(f"{name} must be positive")
    return tuple(numbers)


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
