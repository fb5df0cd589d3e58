"""Polars front end of the Arrow adapters, with the reference's interface
(python/finoptions/polars.py).

A materialised ``polars.DataFrame`` reaches ``finoptions.arrow`` through ``DataFrame.to_arrow()``,
which hands over Polars' own buffers, so the zero-copy and rechunk rules are the Arrow adapters'.
The lazy helpers only check the logical schema and project the pricing columns; they never
collect. Importing this module requires Polars.
"""

from __future__ import annotations

from contextlib import contextmanager
from typing import TYPE_CHECKING, ClassVar

import polars as pl

from . import arrow as _arrow
from .arrow import (
    BufferPolicy,
    CashDividendColumns,
    ContinuousYieldColumn,
    DividendColumns,
    EscrowedCashDividendColumns,
    LsmCallColumns,
    LsmStrikeGroupColumns,
    PreparedLsmCallBatch,
    PreparedLsmStrikeGroups,
)

if TYPE_CHECKING:
    from collections.abc import Iterator

    from .batch_lsm import ExerciseMesh, LsmBatchResult
    from .lsm import Lsm
    from .simulation import CudaExecutor

# Type and buffer errors name no front end, so they are the Arrow classes themselves.
PolarsAdapterTypeError = _arrow.ArrowAdapterTypeError
PolarsBufferError = _arrow.ArrowBufferError


class PolarsSchemaError(_arrow.ArrowSchemaError):
    """A frame lacks a pricing column or has one of another dtype."""

    __slots__ = ()
    frontend: ClassVar[str] = "Polars"


class PolarsContentError(_arrow.ArrowContentError):
    """A frame's content cannot form one pricing request."""

    __slots__ = ()
    frontend: ClassVar[str] = "Polars"


_POLARS_ERRORS = _arrow._Errors(PolarsAdapterTypeError, PolarsSchemaError, PolarsBufferError,  # noqa: SLF001
                                PolarsContentError)


@contextmanager
def _polars_errors() -> Iterator[None]:
    """Re-raise the Arrow schema and content errors of a nested call as their Polars subclasses."""
    try:
        yield
    except _arrow.ArrowSchemaError as error:
        if isinstance(error, PolarsSchemaError):
            raise
        raise PolarsSchemaError(missing=error.missing, mismatches=error.mismatches) from None
    except _arrow.ArrowContentError as error:
        if isinstance(error, PolarsContentError):
            raise
        raise PolarsContentError(violations=error.violations) from None


def _frame(value: object, field: str) -> pl.DataFrame:
    if type(value) is not pl.DataFrame:
        raise PolarsAdapterTypeError(field=field, observed=type(value).__name__,
                                     expected="a materialized polars.DataFrame")
    return value


def _lazy(value: object, field: str) -> pl.LazyFrame:
    if type(value) is not pl.LazyFrame:
        raise PolarsAdapterTypeError(field=field, observed=type(value).__name__, expected="polars.LazyFrame")
    return value


def _polars_schema(columns: tuple[str, ...], dividends: DividendColumns) -> dict[str, pl.DataType]:
    expected: dict[str, pl.DataType] = dict.fromkeys(columns, pl.Float64)
    if type(dividends) is ContinuousYieldColumn:
        expected[dividends.annualized_decimals] = pl.Float64
    elif type(dividends) in (CashDividendColumns, EscrowedCashDividendColumns):
        expected[dividends.times] = pl.List(pl.Float64)
        expected[dividends.amounts] = pl.List(pl.Float64)
    else:
        raise PolarsAdapterTypeError(field="dividends", observed=type(dividends).__name__,
                                     expected="ContinuousYieldColumn, CashDividendColumns, or "
                                              "EscrowedCashDividendColumns")
    return expected


def _check_lazy_schema(observed: pl.Schema, expected: dict[str, pl.DataType]) -> None:
    missing = tuple(name for name in expected if name not in observed)
    mismatches = tuple((name, str(dtype), str(observed[name])) for name, dtype in expected.items()
                       if name in observed and observed[name] != dtype)
    if missing or mismatches:
        raise PolarsSchemaError(missing=missing, mismatches=mismatches)


def select_lsm_call_inputs(frame: pl.LazyFrame, *, columns: LsmCallColumns,
                           dividends: DividendColumns) -> pl.LazyFrame:
    """Project the pricing columns of a lazy query after checking its logical schema (no collect)."""
    lazy = _lazy(frame, "frame")
    if type(columns) is not LsmCallColumns:
        raise PolarsAdapterTypeError(field="columns", observed=type(columns).__name__, expected="LsmCallColumns")
    expected = _polars_schema(columns.ordered(), dividends)
    _check_lazy_schema(lazy.collect_schema(), expected)
    return lazy.select(*expected)


def select_lsm_strike_group_inputs(state_frame: pl.LazyFrame, strike_frame: pl.LazyFrame, *,
                                   state_columns: LsmStrikeGroupColumns, strike_column: str,
                                   dividends: DividendColumns) -> tuple[pl.LazyFrame, pl.LazyFrame]:
    """Project the state and strike axes of two lazy queries after checking their schemas."""
    states, strikes = _lazy(state_frame, "state_frame"), _lazy(strike_frame, "strike_frame")
    if type(state_columns) is not LsmStrikeGroupColumns:
        raise PolarsAdapterTypeError(field="state_columns", observed=type(state_columns).__name__,
                                     expected="LsmStrikeGroupColumns")
    strike_name = _arrow._name(strike_column, field="strike_column")  # noqa: SLF001
    state_schema = _polars_schema(state_columns.ordered(), dividends)
    _check_lazy_schema(states.collect_schema(), state_schema)
    _check_lazy_schema(strikes.collect_schema(), {strike_name: pl.Float64})
    return states.select(*state_schema), strikes.select(strike_name)


def prepare_lsm_call_batch(frame: pl.DataFrame, *, columns: LsmCallColumns, dividends: DividendColumns,
                           buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY) -> PreparedLsmCallBatch:
    """finoptions.arrow.prepare_lsm_call_batch over the frame's Arrow buffers."""
    table = _frame(frame, "frame").to_arrow()
    with _polars_errors():
        return _arrow.prepare_lsm_call_batch(table, columns=columns, dividends=dividends,
                                             buffer_policy=buffer_policy, _errors=_POLARS_ERRORS)


def prepare_lsm_strike_groups(  # noqa: PLR0913 - every compact axis is explicit
    state_frame: pl.DataFrame,
    strike_frame: pl.DataFrame,
    *,
    group_offsets: pl.Series,
    state_columns: LsmStrikeGroupColumns,
    strike_column: str,
    dividends: DividendColumns,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
) -> PreparedLsmStrikeGroups:
    """finoptions.arrow.prepare_lsm_strike_groups over the frames' Arrow buffers."""
    states = _frame(state_frame, "state_frame").to_arrow()
    strikes = _frame(strike_frame, "strike_frame").to_arrow()
    if type(group_offsets) is not pl.Series:
        raise PolarsAdapterTypeError(field="group_offsets", observed=type(group_offsets).__name__,
                                     expected="a materialized polars.Series")
    if group_offsets.n_chunks() > 1 and buffer_policy is BufferPolicy.REQUIRE_ZERO_COPY:
        raise PolarsBufferError(column="group_offsets", policy=buffer_policy,
                                reason="fragmented storage requires an explicit rechunk")
    with _polars_errors():
        return _arrow.prepare_lsm_strike_groups(
            states, strikes, group_offsets=group_offsets.rechunk().to_arrow(), state_columns=state_columns,
            strike_column=strike_column, dividends=dividends, buffer_policy=buffer_policy, _errors=_POLARS_ERRORS)


def lsm_result_frame(result: LsmBatchResult) -> pl.DataFrame:
    """The row-aligned result columns as a Polars frame."""
    return pl.from_arrow(_arrow.lsm_result_table(result))


def price_lsm_call_frame(  # noqa: PLR0913 - every execution contract stays explicit
    frame: pl.DataFrame,
    *,
    columns: LsmCallColumns,
    dividends: DividendColumns,
    mesh: ExerciseMesh,
    executor: CudaExecutor,
    method: Lsm,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
) -> pl.DataFrame:
    """Price one frame's contracts and return the row-aligned result frame."""
    prepared = prepare_lsm_call_batch(frame, columns=columns, dividends=dividends, buffer_policy=buffer_policy)
    return lsm_result_frame(prepared.price(mesh=mesh, executor=executor, method=method))


def price_lsm_strike_group_frames(  # noqa: PLR0913 - every axis and convention is explicit
    state_frame: pl.DataFrame,
    strike_frame: pl.DataFrame,
    *,
    group_offsets: pl.Series,
    state_columns: LsmStrikeGroupColumns,
    strike_column: str,
    dividends: DividendColumns,
    mesh: ExerciseMesh,
    executor: CudaExecutor,
    method: Lsm,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
) -> pl.DataFrame:
    """Price explicit strike groups and return the row-aligned result frame."""
    prepared = prepare_lsm_strike_groups(state_frame, strike_frame, group_offsets=group_offsets,
                                         state_columns=state_columns, strike_column=strike_column,
                                         dividends=dividends, buffer_policy=buffer_policy)
    return lsm_result_frame(prepared.price(mesh=mesh, executor=executor, method=method))


__all__ = [
    "BufferPolicy",
    "CashDividendColumns",
    "ContinuousYieldColumn",
    "DividendColumns",
    "EscrowedCashDividendColumns",
    "LsmCallColumns",
    "LsmStrikeGroupColumns",
    "PolarsAdapterTypeError",
    "PolarsBufferError",
    "PolarsContentError",
    "PolarsSchemaError",
    "PreparedLsmCallBatch",
    "PreparedLsmStrikeGroups",
    "lsm_result_frame",
    "prepare_lsm_call_batch",
    "prepare_lsm_strike_groups",
    "price_lsm_call_frame",
    "price_lsm_strike_group_frames",
    "select_lsm_call_inputs",
    "select_lsm_strike_group_inputs",
]
