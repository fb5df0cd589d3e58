"""Zero-copy Apache Arrow adapters for the batch pricing entries.

The reference materialises Polars frames into its native batch requests (python/finoptions/polars.py:
``prepare_lsm_call_batch`` 332-364, ``prepare_lsm_strike_groups`` 367-431, the result table
486-497). This module gives the same contract over pyarrow tables and record batches, the columnar
format Polars, pandas and DuckDB export without copying: Float64 columns and the children of
List/LargeList(Float64) event columns become read-only NumPy views of the Arrow buffers, which the
batch entries stage to the device as they are. Nothing is cast, sorted, repaired or dropped; a
column split into several chunks is consolidated only under ``BufferPolicy.ALLOW_RECHUNK``.
``finoptions.polars`` reaches these adapters through ``DataFrame.to_arrow()``.

The column specifications, the four error types and their messages follow the reference's
adapter, so that code written against it keeps its meaning; the ragged-contract adapter has no
reference counterpart (the reference's batches take one path count per request).
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import StrEnum
from typing import TYPE_CHECKING, ClassVar, Final

import numpy as np
import numpy.typing as npt
import pyarrow as pa
import pyarrow.compute as pc

from .batch_lsm import (
    BatchDividends,
    CashDividendBatch,
    ContinuousDividendYieldBatch,
    EscrowedCashDividendBatch,
    EscrowedVolatilityConvention,
    LsmBatchResult,
    LsmRaggedContracts,
    LsmStrikeGroups,
    RaggedExerciseTimes,
    price_lsm_call_batch,
    price_lsm_call_grouped_batch,
)
from .dividends import MaturityBoundary, RaggedCashDividends
from .model import DividendPolicy

if TYPE_CHECKING:
    from .batch_lsm import ExerciseMesh
    from .lsm import Lsm
    from .simulation import CudaExecutor

Float64Vector = npt.NDArray[np.float64]

_RESULT_COLUMNS: Final = (
    "prices",
    "sample_standard_deviations",
    "standard_errors",
    "origin_decisions_fitted",
    "origin_exercised",
    "regression_nodes",
    "no_training_support_nodes",
    "insufficient_exercise_support_nodes",
    "minimum_in_the_money_training_paths",
    "maximum_regression_condition_numbers",
    "early_exercise_paths",
    "expiry_paths",
)


class BufferPolicy(StrEnum):
    """What to do with a column whose storage is split into several chunks."""

    REQUIRE_ZERO_COPY = "require_zero_copy"
    ALLOW_RECHUNK = "allow_rechunk"


# ---- errors ----------------------------------------------------------------------------------------
# One family per front end: the Arrow classes here, their Polars subclasses in finoptions.polars.
# `frontend` only names the source in the messages.


@dataclass(slots=True)
class ArrowAdapterTypeError(TypeError):
    """An adapter argument has the wrong runtime type or an invalid column name."""

    field: str
    observed: str
    expected: str

    def __str__(self) -> str:
        """Describe the rejected argument without coercing it."""
        return f"{self.field} must be {self.expected}; observed {self.observed}"


@dataclass(slots=True)
class ArrowSchemaError(ValueError):
    """Pricing columns are missing or have another type than the pricing schema's."""

    missing: tuple[str, ...]
    mismatches: tuple[tuple[str, str, str], ...]
    frontend: ClassVar[str] = "Arrow"

    def __str__(self) -> str:
        """Name the missing and mistyped columns, never their values."""
        return f"invalid {self.frontend} pricing schema: missing={self.missing!r}, mismatches={self.mismatches!r}"


@dataclass(slots=True)
class ArrowBufferError(ValueError):
    """A column's storage cannot be borrowed under the declared buffer policy."""

    column: str
    policy: BufferPolicy
    reason: str

    def __str__(self) -> str:
        """Name the column and the broken storage contract."""
        return f"column {self.column!r} violates {self.policy.value}: {self.reason}"


@dataclass(slots=True)
class ArrowContentError(ValueError):
    """The columns cannot form one pricing request (nulls, empty axes, bad offsets)."""

    violations: tuple[tuple[str, int], ...]
    frontend: ClassVar[str] = "Arrow"

    def __str__(self) -> str:
        """Count the violations, never quote the rows."""
        return f"invalid {self.frontend} pricing content: {self.violations!r}"


@dataclass(frozen=True, slots=True)
class _Errors:
    type_error: type[ArrowAdapterTypeError]
    schema: type[ArrowSchemaError]
    buffer: type[ArrowBufferError]
    content: type[ArrowContentError]


_ARROW_ERRORS: Final = _Errors(ArrowAdapterTypeError, ArrowSchemaError, ArrowBufferError, ArrowContentError)


# ---- column specifications -------------------------------------------------------------------------


def _name(value: object, *, field: str) -> str:
    if type(value) is not str or not value:
        raise ArrowAdapterTypeError(field=field, observed=repr(value), expected="a nonempty plain string")
    return value


def _distinct(names: tuple[str, ...], *, field: str, expected: str) -> None:
    if len(set(names)) != len(names):
        raise ArrowAdapterTypeError(field=field, observed=repr(names), expected=expected)


@dataclass(frozen=True, slots=True)
class LsmCallColumns:
    """Source columns of a row-addressed call batch: one Float64 column per contract field."""

    initial_spot: str
    strike: str
    maturity: str
    rate: str
    volatility: str

    def __post_init__(self) -> None:
        """Five explicit, distinct, nonempty names."""
        names = tuple(_name(getattr(self, f), field=f) for f in ("initial_spot", "strike", "maturity", "rate",
                                                                  "volatility"))
        _distinct(names, field="LSM scalar columns", expected="five distinct column names")

    def ordered(self) -> tuple[str, str, str, str, str]:
        """The native argument order."""
        return (self.initial_spot, self.strike, self.maturity, self.rate, self.volatility)


@dataclass(frozen=True, slots=True)
class LsmStrikeGroupColumns:
    """State columns of a strike-group batch (one row per simulated market state)."""

    initial_spot: str
    maturity: str
    rate: str
    volatility: str

    def __post_init__(self) -> None:
        """Four explicit, distinct, nonempty names."""
        names = tuple(_name(getattr(self, f), field=f) for f in ("initial_spot", "maturity", "rate", "volatility"))
        _distinct(names, field="LSM strike-group state columns", expected="four distinct column names")

    def ordered(self) -> tuple[str, str, str, str]:
        """The native state argument order."""
        return (self.initial_spot, self.maturity, self.rate, self.volatility)


@dataclass(frozen=True, slots=True)
class ContinuousYieldColumn:
    """A Float64 column of continuously compounded annual dividend yields."""

    annualized_decimals: str

    def __post_init__(self) -> None:
        """An explicit source column."""
        _name(self.annualized_decimals, field="annualized_decimals")


@dataclass(frozen=True, slots=True)
class CashDividendColumns:
    """Paired List(Float64) columns of cash-dividend times and amounts, with their conventions."""

    times: str
    amounts: str
    policy: DividendPolicy
    maturity_boundary: MaturityBoundary

    def __post_init__(self) -> None:
        """Distinct event columns and explicit conventions."""
        names = (_name(self.times, field="times"), _name(self.amounts, field="amounts"))
        _distinct(names, field="cash-dividend columns", expected="two distinct column names")
        if type(self.policy) is not DividendPolicy:
            raise ArrowAdapterTypeError(field="policy", observed=type(self.policy).__name__, expected="DividendPolicy")
        if type(self.maturity_boundary) is not MaturityBoundary:
            raise ArrowAdapterTypeError(field="maturity_boundary", observed=type(self.maturity_boundary).__name__,
                                        expected="MaturityBoundary")


@dataclass(frozen=True, slots=True)
class EscrowedCashDividendColumns:
    """Paired List(Float64) cash-event columns for the escrowed approximation."""

    times: str
    amounts: str
    volatility_convention: EscrowedVolatilityConvention
    maturity_boundary: MaturityBoundary

    def __post_init__(self) -> None:
        """Distinct event columns and explicit approximation conventions."""
        names = (_name(self.times, field="times"), _name(self.amounts, field="amounts"))
        _distinct(names, field="escrowed cash-dividend columns", expected="two distinct column names")
        if type(self.volatility_convention) is not EscrowedVolatilityConvention:
            raise ArrowAdapterTypeError(field="volatility_convention",
                                        observed=type(self.volatility_convention).__name__,
                                        expected="EscrowedVolatilityConvention")
        if type(self.maturity_boundary) is not MaturityBoundary:
            raise ArrowAdapterTypeError(field="maturity_boundary", observed=type(self.maturity_boundary).__name__,
                                        expected="MaturityBoundary")


type DividendColumns = ContinuousYieldColumn | CashDividendColumns | EscrowedCashDividendColumns
_DIVIDEND_SPECS: Final = (ContinuousYieldColumn, CashDividendColumns, EscrowedCashDividendColumns)


@dataclass(frozen=True, slots=True)
class LsmRaggedColumns:
    """Source columns of a ragged batch: Float64 contract fields, UInt64 path counts per role, a
    List(Float64) column of exercise times, and optionally a Float64 dividend-yield column."""

    initial_spot: str
    strike: str
    maturity: str
    rate: str
    volatility: str
    training_paths: str
    evaluation_paths: str
    exercise_times: str
    dividend_yield: str | None = None

    def __post_init__(self) -> None:
        """Explicit, distinct, nonempty names."""
        fields = ("initial_spot", "strike", "maturity", "rate", "volatility", "training_paths", "evaluation_paths",
                  "exercise_times")
        names = tuple(_name(getattr(self, f), field=f) for f in fields)
        if self.dividend_yield is not None:
            names = (*names, _name(self.dividend_yield, field="dividend_yield"))
        _distinct(names, field="LSM ragged columns", expected="distinct column names")

    def scalars(self) -> tuple[str, str, str, str, str]:
        """The Float64 contract columns in the native argument order."""
        return (self.initial_spot, self.strike, self.maturity, self.rate, self.volatility)


# ---- prepared requests -------------------------------------------------------------------------------


@dataclass(frozen=True, slots=True, eq=False)
class PreparedLsmCallBatch:
    """A row-addressed call batch whose columns are views of one table's Arrow buffers."""

    initial_spots: Float64Vector
    strikes: Float64Vector
    maturities: Float64Vector
    rates: Float64Vector
    volatilities: Float64Vector
    dividends: BatchDividends

    @property
    def rows(self) -> int:
        """Source-row count."""
        return int(self.initial_spots.size)

    def price(self, *, mesh: ExerciseMesh, executor: CudaExecutor, method: Lsm) -> LsmBatchResult:
        """Price the prepared request on the device (price_lsm_call_batch)."""
        return price_lsm_call_batch(initial_spots=self.initial_spots, strikes=self.strikes,
                                    maturities=self.maturities, rates=self.rates, volatilities=self.volatilities,
                                    dividends=self.dividends, mesh=mesh, executor=executor, method=method)


@dataclass(frozen=True, slots=True, eq=False)
class PreparedLsmStrikeGroups:
    """A strike-group batch whose state, strike and offset axes are views of Arrow buffers."""

    native: LsmStrikeGroups

    def __post_init__(self) -> None:
        """Only the engine's own grouped request."""
        if type(self.native) is not LsmStrikeGroups:
            raise ArrowAdapterTypeError(field="native", observed=type(self.native).__name__, expected="LsmStrikeGroups")

    @property
    def group_count(self) -> int:
        """Independently simulated states."""
        return int(self.native.initial_spots.size)

    @property
    def rows(self) -> int:
        """Strike rows (contracts)."""
        return int(self.native.strikes.size)

    def price(self, *, mesh: ExerciseMesh, executor: CudaExecutor, method: Lsm) -> LsmBatchResult:
        """Price the prepared groups on the device (price_lsm_call_grouped_batch)."""
        return price_lsm_call_grouped_batch(groups=self.native, mesh=mesh, executor=executor, method=method)


# ---- buffers -----------------------------------------------------------------------------------------

def _is_float64_list(t: pa.DataType) -> bool:
    return (pa.types.is_list(t) or pa.types.is_large_list(t)) and t.value_type == pa.float64()


def _check_schema(schema: pa.Schema, expected: dict[str, str], errors: _Errors) -> None:
    """expected maps a column to "float64", "uint64" or "list<float64>" (List or LargeList)."""
    missing = tuple(name for name in expected if name not in schema.names)
    mismatches = []
    for name, kind in expected.items():
        if name not in schema.names:
            continue
        t = schema.field(name).type
        ok = _is_float64_list(t) if kind == "list<float64>" else t == pa.type_for_alias(kind)
        if not ok:
            mismatches.append((name, kind, str(t)))
    if missing or mismatches:
        raise errors.schema(missing=missing, mismatches=tuple(mismatches))


def _one_chunk(column: pa.Array | pa.ChunkedArray, name: str, policy: BufferPolicy, errors: _Errors) -> pa.Array:
    if isinstance(column, pa.Array):
        return column
    if column.num_chunks == 1:
        return column.chunk(0)
    if column.num_chunks == 0:
        return pa.array([], type=column.type)
    if policy is BufferPolicy.REQUIRE_ZERO_COPY:
        raise errors.buffer(column=name, policy=policy, reason="fragmented storage requires an explicit rechunk")
    return column.combine_chunks()


def _vector(array: pa.Array, name: str, policy: BufferPolicy, errors: _Errors, dtype: str) -> np.ndarray:
    """A read-only NumPy view of a null-free primitive Arrow array (no copy)."""
    if array.null_count:
        raise errors.content(violations=((f"null_{name}", int(array.null_count)),))
    try:
        out = array.to_numpy(zero_copy_only=True, writable=False)
    except (pa.ArrowInvalid, pa.ArrowNotImplementedError) as error:
        raise errors.buffer(column=name, policy=policy,
                            reason=f"{dtype} storage cannot be borrowed by NumPy") from error
    if type(out) is not np.ndarray or out.dtype != np.dtype(dtype) or out.ndim != 1 or not out.flags.c_contiguous:
        raise errors.type_error(field=name, observed=f"{type(out).__name__}, {getattr(out, 'dtype', None)}",
                                expected=f"a C-contiguous {dtype} vector")
    return out


def _column(table: pa.Table | pa.RecordBatch, name: str, policy: BufferPolicy, errors: _Errors) -> pa.Array:
    return _one_chunk(table.column(name), name, policy, errors)


def _float64(table, name: str, policy: BufferPolicy, errors: _Errors) -> Float64Vector:
    return _vector(_column(table, name, policy, errors), name, policy, errors, "float64")


def _list_offsets(array: pa.Array) -> np.ndarray:
    """The list's offsets as int64: a view for LargeList, widened (rows + 1 values) for List."""
    offsets = array.offsets.to_numpy(zero_copy_only=True, writable=False)
    return offsets if offsets.dtype == np.int64 else offsets.astype(np.int64)


def _ragged_events(table, times_name: str, amounts_name: str, policy: BufferPolicy,
                   errors: _Errors) -> RaggedCashDividends:
    """Cash events from paired List(Float64) columns: the lists' own offsets (Arrow's layout, with a
    nonzero start for a sliced table) and views of the flattened children."""
    times = _column(table, times_name, policy, errors)
    amounts = _column(table, amounts_name, policy, errors)
    violations = []
    if times.null_count:
        violations.append(("null_cash_time_lists", int(times.null_count)))
    if amounts.null_count:
        violations.append(("null_cash_amount_lists", int(amounts.null_count)))
    mismatched = pc.sum(pc.not_equal(pc.list_value_length(times), pc.list_value_length(amounts))).as_py() or 0
    if mismatched:
        violations.append(("cash_event_length_mismatches", int(mismatched)))
    flat_times, flat_amounts = times.flatten(), amounts.flatten()
    if flat_times.null_count:
        violations.append(("null_cash_times", int(flat_times.null_count)))
    if flat_amounts.null_count:
        violations.append(("null_cash_amounts", int(flat_amounts.null_count)))
    if violations:
        raise errors.content(violations=tuple(violations))
    return RaggedCashDividends(offsets=_list_offsets(times),
                               times=_vector(flat_times, times_name, policy, errors, "float64"),
                               amounts=_vector(flat_amounts, amounts_name, policy, errors, "float64"))


def _dividend_schema(dividends: DividendColumns) -> dict[str, str]:
    if type(dividends) is ContinuousYieldColumn:
        return {dividends.annualized_decimals: "float64"}
    return {dividends.times: "list<float64>", dividends.amounts: "list<float64>"}


def _dividends(table, dividends: DividendColumns, policy: BufferPolicy, errors: _Errors) -> BatchDividends:
    if type(dividends) is ContinuousYieldColumn:
        return ContinuousDividendYieldBatch(
            annualized_decimals=_float64(table, dividends.annualized_decimals, policy, errors))
    events = _ragged_events(table, dividends.times, dividends.amounts, policy, errors)
    if type(dividends) is CashDividendColumns:
        return CashDividendBatch(schedules=events, policy=dividends.policy,
                                 maturity_boundary=dividends.maturity_boundary)
    return EscrowedCashDividendBatch(schedules=events, volatility_convention=dividends.volatility_convention,
                                     maturity_boundary=dividends.maturity_boundary)


# ---- argument checks ---------------------------------------------------------------------------------


def _check_table(value: object, field: str, errors: _Errors) -> None:
    if type(value) not in (pa.Table, pa.RecordBatch):
        raise errors.type_error(field=field, observed=type(value).__name__,
                                expected="a pyarrow.Table or pyarrow.RecordBatch")


def _check_policy(value: object, errors: _Errors) -> None:
    if type(value) is not BufferPolicy:
        raise errors.type_error(field="buffer_policy", observed=type(value).__name__, expected="BufferPolicy")


def _check_dividend_spec(dividends: object, used: tuple[str, ...], field: str, errors: _Errors) -> None:
    if type(dividends) not in _DIVIDEND_SPECS:
        raise errors.type_error(field="dividends", observed=type(dividends).__name__,
                                expected="ContinuousYieldColumn, CashDividendColumns, or EscrowedCashDividendColumns")
    overlap = set(used) & set(_dividend_schema(dividends))
    if overlap:
        raise errors.type_error(field=field, observed=repr(tuple(sorted(overlap))),
                                expected="distinct contract and dividend columns")


# ---- entries -----------------------------------------------------------------------------------------


def prepare_lsm_call_batch(
    table: pa.Table | pa.RecordBatch,
    *,
    columns: LsmCallColumns,
    dividends: DividendColumns,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
    _errors: _Errors = _ARROW_ERRORS,
) -> PreparedLsmCallBatch:
    """Borrow one table as a row-addressed call batch (one contract per row).

    Float64 contract columns, and the children of the List(Float64) cash-event columns, become
    views of the Arrow buffers; a multi-chunk column is consolidated only under ALLOW_RECHUNK.
    """
    _check_table(table, "frame", _errors)
    if type(columns) is not LsmCallColumns:
        raise _errors.type_error(field="columns", observed=type(columns).__name__, expected="LsmCallColumns")
    _check_dividend_spec(dividends, columns.ordered(), "pricing columns", _errors)
    _check_policy(buffer_policy, _errors)
    if table.num_rows == 0:
        raise _errors.content(violations=(("empty_frame", 1),))
    _check_schema(table.schema, {**dict.fromkeys(columns.ordered(), "float64"), **_dividend_schema(dividends)},
                  _errors)
    spot, strike, maturity, rate, vol = (_float64(table, n, buffer_policy, _errors) for n in columns.ordered())
    return PreparedLsmCallBatch(initial_spots=spot, strikes=strike, maturities=maturity, rates=rate,
                                volatilities=vol, dividends=_dividends(table, dividends, buffer_policy, _errors))


def prepare_lsm_strike_groups(  # noqa: PLR0913 - every compact axis is explicit
    state_table: pa.Table | pa.RecordBatch,
    strike_table: pa.Table | pa.RecordBatch,
    *,
    group_offsets: pa.Array | pa.ChunkedArray,
    state_columns: LsmStrikeGroupColumns,
    strike_column: str,
    dividends: DividendColumns,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
    _errors: _Errors = _ARROW_ERRORS,
) -> PreparedLsmStrikeGroups:
    """Borrow a state axis, a strike axis and UInt32 group offsets as one strike-group batch.

    ``state_table`` has one row per simulated market state, ``strike_table`` one row per contract;
    ``group_offsets`` (states + 1 values) cut the strike axis into the states' contiguous groups.
    No grouping, joining, sorting or casting is done.
    """
    _check_table(state_table, "state_frame", _errors)
    _check_table(strike_table, "strike_frame", _errors)
    if not isinstance(group_offsets, (pa.Array, pa.ChunkedArray)):
        raise _errors.type_error(field="group_offsets", observed=type(group_offsets).__name__,
                                 expected="a pyarrow.Array or pyarrow.ChunkedArray")
    if type(state_columns) is not LsmStrikeGroupColumns:
        raise _errors.type_error(field="state_columns", observed=type(state_columns).__name__,
                                 expected="LsmStrikeGroupColumns")
    strike_name = _name(strike_column, field="strike_column")
    _check_dividend_spec(dividends, state_columns.ordered(), "group-state columns", _errors)
    _check_policy(buffer_policy, _errors)
    empty = [(what, 1) for what, t in (("empty_state_frame", state_table), ("empty_strike_frame", strike_table))
             if t.num_rows == 0]
    if empty:
        raise _errors.content(violations=tuple(empty))
    _check_schema(state_table.schema,
                  {**dict.fromkeys(state_columns.ordered(), "float64"), **_dividend_schema(dividends)}, _errors)
    _check_schema(strike_table.schema, {strike_name: "float64"}, _errors)
    if group_offsets.type != pa.uint32():
        raise _errors.schema(missing=(), mismatches=(("group_offsets", "uint32", str(group_offsets.type)),))
    offsets = _vector(_one_chunk(group_offsets, "group_offsets", buffer_policy, _errors), "group_offsets",
                      buffer_policy, _errors, "uint32")
    violations = []
    if offsets.size != state_table.num_rows + 1:
        violations.append(("group_offset_count_mismatch", 1))
    if offsets.size == 0 or int(offsets[0]) != 0 or int(offsets[-1]) != strike_table.num_rows:
        violations.append(("group_offset_boundary_mismatch", 1))
    if offsets.size > 1 and (bad := int(np.count_nonzero(offsets[1:] <= offsets[:-1]))):
        violations.append(("empty_or_reversed_groups", bad))
    if violations:
        raise _errors.content(violations=tuple(violations))
    spot, maturity, rate, vol = (_float64(state_table, n, buffer_policy, _errors) for n in state_columns.ordered())
    return PreparedLsmStrikeGroups(native=LsmStrikeGroups(
        group_offsets=offsets, initial_spots=spot, strikes=_float64(strike_table, strike_name, buffer_policy, _errors),
        maturities=maturity, rates=rate, volatilities=vol,
        dividends=_dividends(state_table, dividends, buffer_policy, _errors)))


def prepare_lsm_ragged_contracts(
    table: pa.Table | pa.RecordBatch,
    *,
    columns: LsmRaggedColumns,
    cash_dividends: tuple[str, str] | None = None,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
) -> LsmRaggedContracts:
    """Borrow one table as a ragged batch (one contract per row, each with its own path counts and
    exercise dates). ``cash_dividends`` names optional paired List(Float64) time / amount columns."""
    errors = _ARROW_ERRORS
    _check_table(table, "frame", errors)
    if type(columns) is not LsmRaggedColumns:
        raise errors.type_error(field="columns", observed=type(columns).__name__, expected="LsmRaggedColumns")
    _check_policy(buffer_policy, errors)
    expected = {**dict.fromkeys(columns.scalars(), "float64"), columns.training_paths: "uint64",
                columns.evaluation_paths: "uint64", columns.exercise_times: "list<float64>"}
    if columns.dividend_yield is not None:
        expected[columns.dividend_yield] = "float64"
    if cash_dividends is not None:
        if (type(cash_dividends) is not tuple or len(cash_dividends) != 2
                or any(type(n) is not str or not n for n in cash_dividends) or cash_dividends[0] == cash_dividends[1]):
            raise errors.type_error(field="cash_dividends", observed=repr(cash_dividends),
                                    expected="a (times, amounts) pair of distinct column names")
        overlap = set(expected) & set(cash_dividends)
        if overlap:
            raise errors.type_error(field="cash_dividends", observed=repr(tuple(sorted(overlap))),
                                    expected="distinct contract and dividend columns")
        expected.update(dict.fromkeys(cash_dividends, "list<float64>"))
    if table.num_rows == 0:
        raise errors.content(violations=(("empty_frame", 1),))
    _check_schema(table.schema, expected, errors)
    spot, strike, maturity, rate, vol = (_float64(table, n, buffer_policy, errors) for n in columns.scalars())
    exercise = _column(table, columns.exercise_times, buffer_policy, errors)
    flat = exercise.flatten()
    if exercise.null_count or flat.null_count:
        raise errors.content(violations=tuple((what, int(n)) for what, n in (
            ("null_exercise_time_lists", exercise.null_count), ("null_exercise_times", flat.null_count)) if n))
    return LsmRaggedContracts(
        initial_spots=spot, strikes=strike, maturities=maturity, rates=rate, volatilities=vol,
        exercise=RaggedExerciseTimes(offsets=_list_offsets(exercise),
                                     times=_vector(flat, columns.exercise_times, buffer_policy, errors, "float64")),
        training_paths=_vector(_column(table, columns.training_paths, buffer_policy, errors), columns.training_paths,
                               buffer_policy, errors, "uint64"),
        evaluation_paths=_vector(_column(table, columns.evaluation_paths, buffer_policy, errors),
                                 columns.evaluation_paths, buffer_policy, errors, "uint64"),
        dividend_yields=None if columns.dividend_yield is None else _float64(table, columns.dividend_yield,
                                                                             buffer_policy, errors),
        cash_dividends=None if cash_dividends is None else _ragged_events(table, *cash_dividends, buffer_policy, errors))


def lsm_result_table(result: LsmBatchResult) -> pa.Table:
    """The row-aligned result columns as an Arrow table (views of the result's arrays)."""
    if type(result) is not LsmBatchResult:
        raise ArrowAdapterTypeError(field="result", observed=type(result).__name__, expected="LsmBatchResult")
    return pa.table({name: pa.array(getattr(result, name)) for name in _RESULT_COLUMNS})


def price_lsm_call_table(  # noqa: PLR0913 - every execution contract stays explicit
    table: pa.Table | pa.RecordBatch,
    *,
    columns: LsmCallColumns,
    dividends: DividendColumns,
    mesh: ExerciseMesh,
    executor: CudaExecutor,
    method: Lsm,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
) -> pa.Table:
    """Price one table's contracts and return the row-aligned result table."""
    prepared = prepare_lsm_call_batch(table, columns=columns, dividends=dividends, buffer_policy=buffer_policy)
    return lsm_result_table(prepared.price(mesh=mesh, executor=executor, method=method))


def price_lsm_strike_group_tables(  # noqa: PLR0913 - every axis and convention is explicit
    state_table: pa.Table | pa.RecordBatch,
    strike_table: pa.Table | pa.RecordBatch,
    *,
    group_offsets: pa.Array | pa.ChunkedArray,
    state_columns: LsmStrikeGroupColumns,
    strike_column: str,
    dividends: DividendColumns,
    mesh: ExerciseMesh,
    executor: CudaExecutor,
    method: Lsm,
    buffer_policy: BufferPolicy = BufferPolicy.REQUIRE_ZERO_COPY,
) -> pa.Table:
    """Price explicit strike groups and return the row-aligned result table."""
    prepared = prepare_lsm_strike_groups(state_table, strike_table, group_offsets=group_offsets,
                                         state_columns=state_columns, strike_column=strike_column,
                                         dividends=dividends, buffer_policy=buffer_policy)
    return lsm_result_table(prepared.price(mesh=mesh, executor=executor, method=method))


__all__ = [
    "ArrowAdapterTypeError",
    "ArrowBufferError",
    "ArrowContentError",
    "ArrowSchemaError",
    "BufferPolicy",
    "CashDividendColumns",
    "ContinuousYieldColumn",
    "DividendColumns",
    "EscrowedCashDividendColumns",
    "LsmCallColumns",
    "LsmRaggedColumns",
    "LsmStrikeGroupColumns",
    "PreparedLsmCallBatch",
    "PreparedLsmStrikeGroups",
    "lsm_result_table",
    "prepare_lsm_call_batch",
    "prepare_lsm_ragged_contracts",
    "prepare_lsm_strike_groups",
    "price_lsm_call_table",
    "price_lsm_strike_group_tables",
]
