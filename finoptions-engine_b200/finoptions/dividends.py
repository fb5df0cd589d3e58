"""Exact ragged cash-dividend schedules (the LSM-path subset of the reference's dividends.py)."""

from __future__ import annotations

from dataclasses import dataclass
from enum import StrEnum
from typing import cast

import numpy as np
import numpy.typing as npt

from . import _native
from .model import InputError

Int64Vector = npt.NDArray[np.int64]
Float64Vector = npt.NDArray[np.float64]
BatchError = _native.BatchError


class MaturityBoundary(StrEnum):
    """Whether an event exactly at option maturity belongs to the model input."""

    STRICTLY_BEFORE = "strictly_before"
    AT_OR_BEFORE = "at_or_before"


def _validate_vector(value: object, *, field: str, dtype: str) -> None:
    if type(value) is not np.ndarray:
        msg = f"{field} must be a plain numpy.ndarray"
        raise InputError(msg)
    array = cast("npt.NDArray[np.generic]", value)
    expected = np.dtype(dtype)
    if array.dtype != expected:
        msg = f"{field} must have dtype {expected}; observed {array.dtype}"
        raise InputError(msg)
    if array.ndim != 1:
        msg = f"{field} must be one-dimensional; observed shape {array.shape}"
        raise InputError(msg)
    if not array.flags.c_contiguous:
        msg = f"{field} must be C-contiguous"
        raise InputError(msg)


@dataclass(frozen=True, slots=True)
class RaggedCashDividends:
    """Arrow-LargeList-style offsets, event times and exact cash amounts (borrowed, not copied).

    Offsets may start above zero when the child arrays are the matching slice of a sliced list.
    """

    offsets: Int64Vector
    times: Float64Vector
    amounts: Float64Vector

    def __post_init__(self) -> None:
        """Fail immediately on malformed layout or invalid event values."""
        _validate_vector(self.offsets, field="offsets", dtype="int64")
        _validate_vector(self.times, field="times", dtype="float64")
        _validate_vector(self.amounts, field="amounts", dtype="float64")
        _native.validate_ragged_cash_dividends_f64(self.offsets, self.times, self.amounts)

    @property
    def rows(self) -> int:
        """Number of option rows."""
        return int(self.offsets.size - 1)

    @property
    def events(self) -> int:
        """Total event count."""
        return int(self.times.size)


__all__ = ["BatchError", "MaturityBoundary", "RaggedCashDividends"]
