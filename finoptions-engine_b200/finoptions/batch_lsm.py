"""Grouped and row-addressed LSM call batches over strict contiguous columns, on a B200.

Same request and result types as the reference's python/finoptions/batch_lsm.py. Every strike in a
group fits its own stopping policy on the group's shared training population and is valued on the
group's shared, disjoint evaluation population (group g uses domains start + g).
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import StrEnum
from typing import Final, cast

import numpy as np
import numpy.typing as npt

from . import _native
from .dividends import MaturityBoundary, RaggedCashDividends
from .lsm import ExerciseTieRule, InsufficientExerciseSupportPolicy, Lsm, LsmError
from .model import DividendPolicy, InputError
from .simulation import RandomStream
from .simulation import CpuExecutor, CudaExecutor, native_executor

Float64Vector = npt.NDArray[np.float64]
Int64Vector = npt.NDArray[np.int64]
UInt32Vector = npt.NDArray[np.uint32]
UInt64Vector = npt.NDArray[np.uint64]
BoolVector = npt.NDArray[np.bool_]

_MAX_U32: Final = (2**32) - 1
_MIN_EVALUATION_PATHS: Final = 2


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
        msg = f"{field} must be C-contiguous; implicit copies are forbidden"
        raise InputError(msg)


class OriginExercise(StrEnum):
    """Whether valuation origin is an explicit common exercise decision."""

    EXCLUDED = "excluded"
    INCLUDED = "included"


class EscrowedVolatilityConvention(StrEnum):
    """Meaning of the volatility column for the escrowed prepaid-forward approximation."""

    PREPAID_FORWARD = "prepaid_forward"
    SPOT_MATCHED_AT_ORIGIN = "spot_matched_at_origin"


@dataclass(frozen=True, slots=True)
class UniformExerciseMesh:
    """Uniform Bermudan base mesh augmented by every exact cash-event time."""

    base_intervals: int
    origin_exercise: OriginExercise

    def __post_init__(self) -> None:
        """Reject empty or inferred meshes and implicit origin semantics."""
        if type(self.base_intervals) is not int or not 1 <= self.base_intervals <= _MAX_U32:
            msg = f"base_intervals must be a plain int in [1, {_MAX_U32}]; observed {self.base_intervals!r}"
            raise InputError(msg)
        if type(self.origin_exercise) is not OriginExercise:
            msg = "origin_exercise must be OriginExercise"
            raise InputError(msg)


@dataclass(frozen=True, slots=True)
class CashDividendExerciseMesh:
    """Exercise only at left limits of strictly pre-expiry deterministic cash events."""


@dataclass(frozen=True, slots=True)
class RaggedExerciseTimes:
    """Row-aligned Arrow-LargeList-style exact exercise times."""

    offsets: Int64Vector
    times: Float64Vector

    def __post_init__(self) -> None:
        """Reject malformed, invalid, duplicate or unordered opportunities without copying."""
        _validate_vector(self.offsets, field="exercise offsets", dtype="int64")
        _validate_vector(self.times, field="exercise times", dtype="float64")
        _native.validate_ragged_exercise_times_f64(self.offsets, self.times)

    @property
    def rows(self) -> int:
        """Schedule-row count."""
        return int(self.offsets.size - 1)

    @property
    def events(self) -> int:
        """Total opportunity count."""
        return int(self.times.size)


@dataclass(frozen=True, slots=True)
class ExplicitExerciseMesh:
    """Exact row-aligned pre-expiry Bermudan opportunities; cash times are transition nodes only."""

    schedules: RaggedExerciseTimes
    origin_exercise: OriginExercise

    def __post_init__(self) -> None:
        """Reject duck-typed schedules and implicit origin semantics."""
        if type(self.schedules) is not RaggedExerciseTimes:
            msg = "schedules must be RaggedExerciseTimes"
            raise InputError(msg)
        if type(self.origin_exercise) is not OriginExercise:
            msg = "origin_exercise must be OriginExercise"
            raise InputError(msg)


@dataclass(frozen=True, slots=True)
class ContinuousDividendYieldBatch:
    """One constant nonnegative proportional yield per row or group."""

    annualized_decimals: Float64Vector

    def __post_init__(self) -> None:
        """Require one borrowable float64 vector."""
        _validate_vector(self.annualized_decimals, field="annualized_decimals", dtype="float64")


@dataclass(frozen=True, slots=True)
class CashDividendBatch:
    """Exact cash schedules with explicit jump policy and maturity boundary."""

    schedules: RaggedCashDividends
    policy: DividendPolicy
    maturity_boundary: MaturityBoundary

    def __post_init__(self) -> None:
        """Reject duck-typed schedules and implicit conventions."""
        if type(self.schedules) is not RaggedCashDividends:
            raise InputError("schedules must be RaggedCashDividends")
        if type(self.policy) is not DividendPolicy:
            raise InputError("policy must be DividendPolicy")
        if type(self.maturity_boundary) is not MaturityBoundary:
            raise InputError("maturity_boundary must be MaturityBoundary")


@dataclass(frozen=True, slots=True)
class EscrowedCashDividendBatch:
    """Escrowed approximation: risky prepaid forward plus deterministic prepaid cash."""

    schedules: RaggedCashDividends
    volatility_convention: EscrowedVolatilityConvention
    maturity_boundary: MaturityBoundary

    def __post_init__(self) -> None:
        """Reject duck-typed schedules and any implicit volatility interpretation."""
        if type(self.schedules) is not RaggedCashDividends:
            raise InputError("schedules must be RaggedCashDividends")
        if type(self.volatility_convention) is not EscrowedVolatilityConvention:
            raise InputError("volatility_convention must be EscrowedVolatilityConvention")
        if type(self.maturity_boundary) is not MaturityBoundary:
            raise InputError("maturity_boundary must be MaturityBoundary")


type BatchDividends = ContinuousDividendYieldBatch | CashDividendBatch | EscrowedCashDividendBatch
type ExerciseMesh = UniformExerciseMesh | CashDividendExerciseMesh | ExplicitExerciseMesh
_DIVIDEND_TYPES: Final = (ContinuousDividendYieldBatch, CashDividendBatch, EscrowedCashDividendBatch)
_MESH_TYPES: Final = (UniformExerciseMesh, CashDividendExerciseMesh, ExplicitExerciseMesh)


def _mesh_arguments(mesh: ExerciseMesh) -> tuple:
    if type(mesh) is UniformExerciseMesh:
        return ("uniform", mesh.base_intervals, mesh.origin_exercise.value, None, None)
    if type(mesh) is CashDividendExerciseMesh:
        return ("cash_dividend_dates", None, None, None, None)
    if type(mesh) is ExplicitExerciseMesh:
        return ("explicit_times", None, mesh.origin_exercise.value, mesh.schedules.offsets, mesh.schedules.times)
    msg = "exercise mesh changed type after request validation"
    raise LsmError(msg)


def _validate_mesh(mesh: object, dividends: object, expected_rows: int) -> None:
    if type(mesh) not in _MESH_TYPES:
        msg = "mesh must be UniformExerciseMesh, CashDividendExerciseMesh, or ExplicitExerciseMesh"
        raise InputError(msg)
    if type(mesh) is ExplicitExerciseMesh and mesh.schedules.rows != expected_rows:
        msg = f"explicit exercise schedules have {mesh.schedules.rows} rows; expected {expected_rows}"
        raise InputError(msg)
    if type(mesh) is CashDividendExerciseMesh and type(dividends) is ContinuousDividendYieldBatch:
        msg = "CashDividendExerciseMesh requires cash-dividend inputs"
        raise InputError(msg)


def _validate_executor_method(executor: object, method: object, what: str) -> None:
    if type(executor) not in (CudaExecutor, CpuExecutor):
        msg = "executor must be CudaExecutor"
        raise InputError(msg)
    if type(method) is not Lsm:
        msg = "method must be Lsm"
        raise InputError(msg)
    if method.evaluation_paths < _MIN_EVALUATION_PATHS:
        msg = f"{what} requires at least two independent evaluation paths"
        raise InputError(msg)


@dataclass(frozen=True, slots=True)
class LsmStrikeGroups:
    """Compact simulation states, each with one or more row-ordered strikes.

    ``group_offsets`` are contiguous uint32 strike-row boundaries; spot, maturity, rate,
    volatility and dividends have one entry per group, ``strikes`` one entry per contract.
    """

    group_offsets: UInt32Vector
    initial_spots: Float64Vector
    strikes: Float64Vector
    maturities: Float64Vector
    rates: Float64Vector
    volatilities: Float64Vector
    dividends: BatchDividends

    def __post_init__(self) -> None:
        """Require directly borrowable compact columns; the engine revalidates all values."""
        _validate_vector(self.group_offsets, field="group_offsets", dtype="uint32")
        for name, values in (
            ("initial_spots", self.initial_spots),
            ("strikes", self.strikes),
            ("maturities", self.maturities),
            ("rates", self.rates),
            ("volatilities", self.volatilities),
        ):
            _validate_vector(values, field=name, dtype="float64")
        if type(self.dividends) not in _DIVIDEND_TYPES:
            msg = "dividends must be ContinuousDividendYieldBatch, CashDividendBatch, or EscrowedCashDividendBatch"
            raise InputError(msg)


_RESULT_FIELDS: Final = (
    ("prices", "float64"),
    ("sample_standard_deviations", "float64"),
    ("standard_errors", "float64"),
    ("origin_decisions_fitted", "bool"),
    ("origin_exercised", "bool"),
    ("regression_nodes", "uint32"),
    ("no_training_support_nodes", "uint32"),
    ("insufficient_exercise_support_nodes", "uint32"),
    ("minimum_in_the_money_training_paths", "uint32"),
    ("maximum_regression_condition_numbers", "float64"),
    ("early_exercise_paths", "uint32"),
    ("expiry_paths", "uint32"),
)


@dataclass(frozen=True, slots=True, eq=False)
class LsmBatchResult:
    """Immutable row-ordered prices, sampling error, policy support and stopping counts."""

    prices: Float64Vector
    sample_standard_deviations: Float64Vector
    standard_errors: Float64Vector
    origin_decisions_fitted: BoolVector
    origin_exercised: BoolVector
    regression_nodes: UInt32Vector
    no_training_support_nodes: UInt32Vector
    insufficient_exercise_support_nodes: UInt32Vector
    minimum_in_the_money_training_paths: UInt32Vector
    maximum_regression_condition_numbers: Float64Vector
    early_exercise_paths: UInt32Vector
    expiry_paths: UInt32Vector

    def __post_init__(self) -> None:
        """Reject manually assembled outputs outside the immutable column contract."""
        rows = int(self.prices.size)
        for name, dtype in _RESULT_FIELDS:
            values = getattr(self, name)
            _validate_vector(values, field=name, dtype=dtype)
            if values.size != rows:
                msg = f"{name} has {values.size} rows; expected {rows}"
                raise InputError(msg)
            if values.flags.writeable:
                msg = f"{name} must be immutable"
                raise InputError(msg)

    @property
    def rows(self) -> int:
        """Priced contract count."""
        return int(self.prices.size)


def _freeze(raw: tuple) -> LsmBatchResult:
    columns = {}
    for (name, _), values in zip(_RESULT_FIELDS, raw, strict=True):
        values.flags.writeable = False
        columns[name] = values
    return LsmBatchResult(**columns)


def _check_partition(result: LsmBatchResult, evaluation_paths: int, what: str) -> LsmBatchResult:
    stopping = result.early_exercise_paths.astype(np.uint64) + result.expiry_paths.astype(np.uint64)
    if np.any(stopping != evaluation_paths):
        msg = f"native {what} stopping counts do not partition evaluation paths"
        raise LsmError(msg)
    return result


def _method_arguments(mesh: ExerciseMesh, executor: object, method: Lsm) -> tuple:
    return (
        *_mesh_arguments(mesh),
        None if executor is None else native_executor(executor),
        method.training_paths,
        method.evaluation_paths,
        method.training_stream.seed,
        method.training_stream.domain,
        method.evaluation_stream.seed,
        method.evaluation_stream.domain,
        method.polynomial_degree,
        method.rank_tolerance,
        method.condition_limit,
        method.tie_rule.value,
        method.insufficient_exercise_support.value,
    )


def price_lsm_call_grouped_batch(
    *,
    groups: LsmStrikeGroups,
    mesh: ExerciseMesh,
    executor: CudaExecutor,
    method: Lsm,
) -> LsmBatchResult:
    """Price strike groups while simulating each declared market state exactly once.

    Each strike fits its own stopping policy on the shared group training population and is valued
    out of sample on the shared, disjoint evaluation population. Arrays are borrowed; nothing is
    cast, sorted, repaired or inferred, and no failure falls back to another method or device.
    """
    if type(groups) is not LsmStrikeGroups:
        raise InputError("groups must be LsmStrikeGroups")
    _validate_executor_method(executor, method, "grouped batched LSM")
    return _grouped_call(groups, mesh, executor, method)


def validate_lsm_call_grouped_batch(*, groups: LsmStrikeGroups, mesh: ExerciseMesh, method: Lsm) -> None:
    """Every check price_lsm_call_grouped_batch makes on the whole request before it plans any
    group (method, columns, the stream domain ranges over every group, mesh domain), with the same
    typed errors, and without touching a device. A caller that prices a batch in shards runs it on
    the whole request first: each shard sees fewer groups and shifted domains, so the shards alone
    cannot see, e.g., training and evaluation domain ranges that overlap."""
    if type(groups) is not LsmStrikeGroups:
        raise InputError("groups must be LsmStrikeGroups")
    if type(method) is not Lsm:
        raise InputError("method must be Lsm")
    if method.evaluation_paths < _MIN_EVALUATION_PATHS:
        raise InputError("grouped batched LSM requires at least two independent evaluation paths")
    _grouped_call(groups, mesh, None, method)


def _grouped_call(groups: LsmStrikeGroups, mesh: ExerciseMesh, executor: object, method: Lsm) -> LsmBatchResult | None:
    _validate_mesh(mesh, groups.dividends, int(groups.initial_spots.size))
    common = (groups.group_offsets, groups.initial_spots, groups.strikes, groups.maturities, groups.rates,
              groups.volatilities)
    tail = _method_arguments(mesh, executor, method)
    d = groups.dividends
    if type(d) is ContinuousDividendYieldBatch:
        raw = _native.price_lsm_call_grouped_batch_continuous_yield_f64(*common, d.annualized_decimals, *tail)
    elif type(d) is CashDividendBatch:
        raw = _native.price_lsm_call_grouped_batch_cash_dividends_f64(
            *common, d.schedules.offsets, d.schedules.times, d.schedules.amounts, d.policy.value,
            d.maturity_boundary.value, *tail)
    elif type(d) is EscrowedCashDividendBatch:
        raw = _native.price_lsm_call_grouped_batch_escrowed_cash_dividends_f64(
            *common, d.schedules.offsets, d.schedules.times, d.schedules.amounts, d.volatility_convention.value,
            d.maturity_boundary.value, *tail)
    else:
        raise LsmError("group dividends changed type after request validation")
    if executor is None:
        return None
    return _check_partition(_freeze(raw), method.evaluation_paths, "grouped LSM")


def price_lsm_call_batch(  # noqa: PLR0913 - each financial column is independently typed
    *,
    initial_spots: Float64Vector,
    strikes: Float64Vector,
    maturities: Float64Vector,
    rates: Float64Vector,
    volatilities: Float64Vector,
    dividends: BatchDividends,
    mesh: ExerciseMesh,
    executor: CudaExecutor,
    method: Lsm,
) -> LsmBatchResult:
    """Price constant-parameter Bermudan calls, one independent population pair per row.

    Row r uses ``training_stream.domain + r`` and ``evaluation_stream.domain + r``.
    """
    for name, values in (
        ("initial_spots", initial_spots),
        ("strikes", strikes),
        ("maturities", maturities),
        ("rates", rates),
        ("volatilities", volatilities),
    ):
        _validate_vector(values, field=name, dtype="float64")
    if type(dividends) not in _DIVIDEND_TYPES:
        msg = "dividends must be ContinuousDividendYieldBatch, CashDividendBatch, or EscrowedCashDividendBatch"
        raise InputError(msg)
    _validate_mesh(mesh, dividends, int(initial_spots.size))
    _validate_executor_method(executor, method, "batched LSM")
    common = (initial_spots, strikes, maturities, rates, volatilities)
    tail = _method_arguments(mesh, executor, method)
    if type(dividends) is ContinuousDividendYieldBatch:
        raw = _native.price_lsm_call_batch_continuous_yield_f64(*common, dividends.annualized_decimals, *tail)
    elif type(dividends) is CashDividendBatch:
        s = dividends.schedules
        raw = _native.price_lsm_call_batch_cash_dividends_f64(
            *common, s.offsets, s.times, s.amounts, dividends.policy.value, dividends.maturity_boundary.value, *tail)
    else:
        s = dividends.schedules
        raw = _native.price_lsm_call_batch_escrowed_cash_dividends_f64(
            *common, s.offsets, s.times, s.amounts, dividends.volatility_convention.value,
            dividends.maturity_boundary.value, *tail)
    return _check_partition(_freeze(raw), method.evaluation_paths, "batched LSM")


# ---- ragged batches (no reference counterpart) ---------------------------------------------------


@dataclass(frozen=True, slots=True)
class LsmRaggedContracts:
    """Independent call contracts, each with its own training and evaluation path count.

    Every column has one entry per contract. Row r is priced like a one-row explicit-mesh batch with
    domains ``training_stream.domain + r`` / ``evaluation_stream.domain + r``: its exercise times,
    a continuous yield (``dividend_yields``, optional) and/or cash dividends (optional) merged into
    its exact mesh. The reference's batch methods take one path count per request.
    """

    initial_spots: Float64Vector
    strikes: Float64Vector
    maturities: Float64Vector
    rates: Float64Vector
    volatilities: Float64Vector
    exercise: RaggedExerciseTimes
    training_paths: UInt64Vector
    evaluation_paths: UInt64Vector
    dividend_yields: Float64Vector | None = None
    cash_dividends: RaggedCashDividends | None = None

    def __post_init__(self) -> None:
        """Require directly borrowable columns; the engine validates every value."""
        for name in ("initial_spots", "strikes", "maturities", "rates", "volatilities"):
            _validate_vector(getattr(self, name), field=name, dtype="float64")
        for name in ("training_paths", "evaluation_paths"):
            _validate_vector(getattr(self, name), field=name, dtype="uint64")
        if self.dividend_yields is not None:
            _validate_vector(self.dividend_yields, field="dividend_yields", dtype="float64")
        if type(self.exercise) is not RaggedExerciseTimes:
            raise InputError("exercise must be RaggedExerciseTimes")
        if self.cash_dividends is not None and type(self.cash_dividends) is not RaggedCashDividends:
            raise InputError("cash_dividends must be RaggedCashDividends")

    @property
    def rows(self) -> int:
        """Contract count."""
        return int(self.initial_spots.size)

    def mesh_nodes(self) -> int:
        """Nodes of every row's exact mesh (origin, merged exercise and cash times, maturity)."""
        total = 0
        ex, cash = self.exercise, self.cash_dividends
        for r in range(self.rows):
            times = ex.times[ex.offsets[r] - ex.offsets[0]:ex.offsets[r + 1] - ex.offsets[0]]
            if cash is not None:
                c = cash.times[cash.offsets[r] - cash.offsets[0]:cash.offsets[r + 1] - cash.offsets[0]]
                times = np.union1d(times, c)
            total += int(np.unique(times[times < self.maturities[r]]).size) + 2
        return total


@dataclass(frozen=True, slots=True, eq=False)
class LsmRaggedGreeks:
    """Fixed-policy pathwise Greeks of a ragged batch: per row delta and vega; dPrice/dL for every
    node of row r's mesh at ``log_discount_sensitivities[log_discount_offsets[r]:log_discount_offsets[r + 1]]``
    (L the log discounts -r t); dPrice/dD per cash event, aligned with the cash-dividend times."""

    delta: Float64Vector
    vega: Float64Vector
    log_discount_sensitivities: Float64Vector
    log_discount_offsets: Int64Vector
    dividend_sensitivities: Float64Vector


def _ragged_arguments(contracts: LsmRaggedContracts, origin_exercise: OriginExercise, dividend_policy: DividendPolicy,
                      maturity_boundary: MaturityBoundary, executor: object, training_stream: RandomStream,
                      evaluation_stream: RandomStream, insufficient_exercise_support: InsufficientExerciseSupportPolicy,
                      polynomial_degree: int, rank_tolerance: float, condition_limit: float,
                      tie_rule: ExerciseTieRule) -> tuple:
    if type(contracts) is not LsmRaggedContracts:
        raise InputError("contracts must be LsmRaggedContracts")
    cash = contracts.cash_dividends
    return (
        contracts.initial_spots, contracts.strikes, contracts.maturities, contracts.rates, contracts.volatilities,
        contracts.dividend_yields, None if cash is None else cash.offsets, None if cash is None else cash.times,
        None if cash is None else cash.amounts, dividend_policy.value, maturity_boundary.value,
        contracts.exercise.offsets, contracts.exercise.times, origin_exercise.value, contracts.training_paths,
        contracts.evaluation_paths, None if executor is None else native_executor(executor), training_stream.seed,
        training_stream.domain,
        evaluation_stream.seed, evaluation_stream.domain, polynomial_degree, rank_tolerance, condition_limit,
        tie_rule.value, insufficient_exercise_support.value,
    )


def price_lsm_call_ragged(  # noqa: PLR0913 - method settings stay explicit keywords
    *,
    contracts: LsmRaggedContracts,
    origin_exercise: OriginExercise,
    executor: CudaExecutor,
    training_stream: RandomStream,
    evaluation_stream: RandomStream,
    insufficient_exercise_support: InsufficientExerciseSupportPolicy,
    dividend_policy: DividendPolicy = DividendPolicy.LIQUIDATOR,
    maturity_boundary: MaturityBoundary = MaturityBoundary.STRICTLY_BEFORE,
    polynomial_degree: int = 4,
    rank_tolerance: float = 1.0e-12,
    condition_limit: float = 1.0e8,
    tie_rule: ExerciseTieRule = ExerciseTieRule.STRICTLY_GREATER,
) -> LsmBatchResult:
    """Price independent contracts with their own path counts in one batch."""
    raw = _native.price_lsm_call_ragged_f64(*_ragged_arguments(
        contracts, origin_exercise, dividend_policy, maturity_boundary, executor, training_stream, evaluation_stream,
        insufficient_exercise_support, polynomial_degree, rank_tolerance, condition_limit, tie_rule))
    return _freeze(raw)


def validate_lsm_call_ragged(  # noqa: PLR0913 - method settings stay explicit keywords
    *,
    contracts: LsmRaggedContracts,
    origin_exercise: OriginExercise,
    training_stream: RandomStream,
    evaluation_stream: RandomStream,
    insufficient_exercise_support: InsufficientExerciseSupportPolicy,
    dividend_policy: DividendPolicy = DividendPolicy.LIQUIDATOR,
    maturity_boundary: MaturityBoundary = MaturityBoundary.STRICTLY_BEFORE,
    polynomial_degree: int = 4,
    rank_tolerance: float = 1.0e-12,
    condition_limit: float = 1.0e8,
    tie_rule: ExerciseTieRule = ExerciseTieRule.STRICTLY_GREATER,
) -> None:
    """Every check price_lsm_call_ragged makes on the whole request, without touching a device."""
    _native.price_lsm_call_ragged_f64(*_ragged_arguments(
        contracts, origin_exercise, dividend_policy, maturity_boundary, None, training_stream, evaluation_stream,
        insufficient_exercise_support, polynomial_degree, rank_tolerance, condition_limit, tie_rule))


def price_lsm_call_ragged_greeks(  # noqa: PLR0913 - method settings stay explicit keywords
    *,
    contracts: LsmRaggedContracts,
    origin_exercise: OriginExercise,
    executor: CudaExecutor,
    training_stream: RandomStream,
    evaluation_stream: RandomStream,
    insufficient_exercise_support: InsufficientExerciseSupportPolicy,
    dividend_policy: DividendPolicy = DividendPolicy.LIQUIDATOR,
    maturity_boundary: MaturityBoundary = MaturityBoundary.STRICTLY_BEFORE,
    polynomial_degree: int = 4,
    rank_tolerance: float = 1.0e-12,
    condition_limit: float = 1.0e8,
    tie_rule: ExerciseTieRule = ExerciseTieRule.STRICTLY_GREATER,
) -> tuple[LsmBatchResult, LsmRaggedGreeks]:
    """Price independent contracts and their fixed-policy adjoint Greeks in the same pass."""
    raw, delta, vega, d_l, offsets, d_d = _native.price_lsm_call_ragged_f64(
        *_ragged_arguments(contracts, origin_exercise, dividend_policy, maturity_boundary, executor, training_stream,
                           evaluation_stream, insufficient_exercise_support, polynomial_degree, rank_tolerance,
                           condition_limit, tie_rule),
        log_discount_nodes=contracts.mesh_nodes())
    for array in (delta, vega, d_l, offsets, d_d):
        array.flags.writeable = False
    return _freeze(raw), LsmRaggedGreeks(delta=delta, vega=vega, log_discount_sensitivities=d_l,
                                         log_discount_offsets=offsets, dividend_sensitivities=d_d)


__all__ = [
    "BatchDividends",
    "CashDividendBatch",
    "CashDividendExerciseMesh",
    "ContinuousDividendYieldBatch",
    "EscrowedCashDividendBatch",
    "EscrowedVolatilityConvention",
    "ExerciseMesh",
    "ExplicitExerciseMesh",
    "LsmBatchResult",
    "LsmRaggedContracts",
    "LsmRaggedGreeks",
    "LsmStrikeGroups",
    "OriginExercise",
    "RaggedExerciseTimes",
    "UniformExerciseMesh",
    "price_lsm_call_batch",
    "price_lsm_call_grouped_batch",
    "price_lsm_call_ragged",
    "price_lsm_call_ragged_greeks",
    "validate_lsm_call_grouped_batch",
    "validate_lsm_call_ragged",
]
