"""Independent-policy least-squares Monte Carlo for explicitly scheduled calls, on a B200.

Same specification and result types as the reference's python/finoptions/lsm.py. ``price_lsm_call``
fits the stopping policy on the training population and values it only on the independent
evaluation population; the whole pass runs on the device behind the C ABI.
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import StrEnum
from math import isfinite
from typing import Final

from . import _native
from ._abi import (
    FO_DIAG_INSUFFICIENT_SUPPORT,
    FO_DIAG_NO_IN_THE_MONEY_PATHS,
    FO_DIAG_ORIGIN_DECISION,
    FO_DIAG_REGRESSION,
)
from .model import (
    ConstantVolatility,
    CumulativeDividendYieldCurve,
    DividendPolicy,
    EventSchedule,
    InputError,
    LogDiscountCurve,
)
from .simulation import CpuExecutor, CudaExecutor, RandomStream, native_executor

LsmError = _native.LsmError
_MAX_PATHS: Final = (2**32) - 1
_MAX_POLYNOMIAL_DEGREE: Final = 4


class ExerciseTieRule(StrEnum):
    """Decision when intrinsic value and fitted continuation compare equal."""

    STRICTLY_GREATER = "strictly_greater"
    GREATER_OR_EQUAL = "greater_or_equal"


class InsufficientExerciseSupportPolicy(StrEnum):
    """Stopping rule when in-the-money training rows cannot identify the polynomial basis."""

    FAIL = "fail"
    CONTINUE = "continue"


def _validate_random_streams(training: RandomStream, evaluation: RandomStream) -> None:
    if type(training) is not RandomStream:
        msg = "training_stream must be RandomStream"
        raise InputError(msg)
    if type(evaluation) is not RandomStream:
        msg = "evaluation_stream must be RandomStream"
        raise InputError(msg)
    if training.domain == evaluation.domain:
        msg = f"training_stream and evaluation_stream must use different domains; both use {training.domain}"
        raise InputError(msg)


@dataclass(frozen=True, slots=True)
class Lsm:
    """Complete simulation / regression identity of one independent-policy LSM estimator."""

    training_paths: int
    evaluation_paths: int
    training_stream: RandomStream
    evaluation_stream: RandomStream
    insufficient_exercise_support: InsufficientExerciseSupportPolicy
    polynomial_degree: int = 4
    rank_tolerance: float = 1.0e-12
    condition_limit: float = 1.0e8
    tie_rule: ExerciseTieRule = ExerciseTieRule.STRICTLY_GREATER

    def __post_init__(self) -> None:
        """Reject inferred types, unsupported degrees, invalid gates and reused domains."""
        for name, value in (("training_paths", self.training_paths), ("evaluation_paths", self.evaluation_paths)):
            if type(value) is not int or not 1 <= value <= _MAX_PATHS:
                msg = f"{name} must be a plain int in [1, {_MAX_PATHS}]; observed {value!r}"
                raise InputError(msg)
        _validate_random_streams(self.training_stream, self.evaluation_stream)
        if type(self.insufficient_exercise_support) is not InsufficientExerciseSupportPolicy:
            msg = (
                "insufficient_exercise_support must be InsufficientExerciseSupportPolicy; "
                f"observed {type(self.insufficient_exercise_support).__name__}"
            )
            raise InputError(msg)
        if type(self.polynomial_degree) is not int or not 0 <= self.polynomial_degree <= _MAX_POLYNOMIAL_DEGREE:
            msg = (
                f"polynomial_degree must be a plain int in [0, {_MAX_POLYNOMIAL_DEGREE}]; "
                f"observed {self.polynomial_degree!r}"
            )
            raise InputError(msg)
        if type(self.rank_tolerance) is not float or not isfinite(self.rank_tolerance) or not (
            0.0 < self.rank_tolerance < 1.0
        ):
            msg = (
                "rank_tolerance must be a finite plain float strictly between 0 and 1; "
                f"observed {self.rank_tolerance!r}"
            )
            raise InputError(msg)
        maximum = 1.0 / self.rank_tolerance
        if type(self.condition_limit) is not float or not isfinite(self.condition_limit) or not (
            1.0 <= self.condition_limit <= maximum
        ):
            msg = f"condition_limit must be a finite plain float in [1, {maximum}]; observed {self.condition_limit!r}"
            raise InputError(msg)
        if type(self.tie_rule) is not ExerciseTieRule:
            msg = f"tie_rule must be ExerciseTieRule; observed {type(self.tie_rule).__name__}"
            raise InputError(msg)


@dataclass(frozen=True, slots=True)
class OriginDecisionDiagnostics:
    """Common valuation-origin decision fitted from the training continuation mean."""

    node: int
    exercise: bool
    estimated_continuation: float


@dataclass(frozen=True, slots=True)
class NoInTheMoneyPathsDiagnostics:
    """Training had no in-the-money state at this exercise node."""

    node: int


@dataclass(frozen=True, slots=True)
class InsufficientExerciseSupportDiagnostics:
    """Declared continuation at a node whose training population cannot identify the basis."""

    node: int
    in_the_money_paths: int
    required_paths: int


@dataclass(frozen=True, slots=True)
class RegressionFitDiagnostics:
    """Accepted continuation regression and its numerical diagnostics."""

    node: int
    in_the_money_paths: int
    observations: int
    columns: int
    rank: int
    condition_number: float
    predictor_mean: float
    predictor_scale: float


type ExerciseFitDiagnostics = (
    OriginDecisionDiagnostics
    | NoInTheMoneyPathsDiagnostics
    | InsufficientExerciseSupportDiagnostics
    | RegressionFitDiagnostics
)


@dataclass(frozen=True, slots=True)
class LsmResult:
    """Independent mean payoff, sampling error, stopping counts and per-node fit diagnostics."""

    price: float
    paths: int
    sample_standard_deviation: float | None
    standard_error: float | None
    observation_nodes: tuple[int, ...]
    exercise_counts: tuple[int, ...]
    fit_diagnostics: tuple[ExerciseFitDiagnostics, ...]


def _required[T](value: T | None, *, field: str) -> T:
    if value is None:
        msg = f"native LSM result omitted required {field}"
        raise LsmError(msg)
    return value


# Regression rows are most of a result; their frozen records are filled through the slot
# descriptors (the same objects the constructor makes, without its per-field frozen-setattr path).
_new_record = object.__new__
(_set_node, _set_itm, _set_observations, _set_columns, _set_rank, _set_condition, _set_mean,
 _set_scale) = (getattr(RegressionFitDiagnostics, name).__set__ for name in (
    "node", "in_the_money_paths", "observations", "columns", "rank", "condition_number", "predictor_mean",
    "predictor_scale"))


_OTHER_KINDS = frozenset((FO_DIAG_ORIGIN_DECISION, FO_DIAG_NO_IN_THE_MONEY_PATHS, FO_DIAG_INSUFFICIENT_SUPPORT))


def _fit_records(rows: list[tuple]) -> tuple[ExerciseFitDiagnostics, ...]:
    """The records of native diagnostic rows (CallResult.rows()): the records _fit_diagnostic makes
    from the NativeLsmResult tuples of the same rows, in one pass."""
    out = []
    append = out.append
    for node, kind, exercise, continuation, itm, observations, columns, rank, condition, mean, scale in rows:
        if kind == FO_DIAG_REGRESSION or kind not in _OTHER_KINDS:  # unknown kinds read as regression rows
            record = _new_record(RegressionFitDiagnostics)
            _set_node(record, node)
            _set_itm(record, itm)
            _set_observations(record, observations)
            _set_columns(record, columns)
            _set_rank(record, rank)
            _set_condition(record, condition)
            _set_mean(record, mean)
            _set_scale(record, scale)
            append(record)
        elif kind == FO_DIAG_ORIGIN_DECISION:
            append(OriginDecisionDiagnostics(node=node, exercise=bool(exercise), estimated_continuation=continuation))
        elif kind == FO_DIAG_NO_IN_THE_MONEY_PATHS:
            append(NoInTheMoneyPathsDiagnostics(node=node))
        else:
            append(InsufficientExerciseSupportDiagnostics(node=node, in_the_money_paths=itm, required_paths=columns))
    return tuple(out)


def _fit_diagnostic(raw: tuple) -> ExerciseFitDiagnostics:
    (node, kind, exercise, continuation, itm, observations, columns, rank, condition, mean, scale) = raw
    if kind == "regression" and None not in (itm, observations, columns, rank, condition, mean, scale):
        record = _new_record(RegressionFitDiagnostics)
        _set_node(record, node)
        _set_itm(record, itm)
        _set_observations(record, observations)
        _set_columns(record, columns)
        _set_rank(record, rank)
        _set_condition(record, condition)
        _set_mean(record, mean)
        _set_scale(record, scale)
        return record
    if kind == "origin_decision":
        return OriginDecisionDiagnostics(
            node=node,
            exercise=_required(exercise, field="origin exercise decision"),
            estimated_continuation=_required(continuation, field="origin continuation estimate"),
        )
    if kind == "no_in_the_money_paths":
        return NoInTheMoneyPathsDiagnostics(node=node)
    if kind == "insufficient_exercise_support":
        return InsufficientExerciseSupportDiagnostics(
            node=node,
            in_the_money_paths=_required(itm, field="in-the-money path count"),
            required_paths=_required(columns, field="required regression path count"),
        )
    if kind == "regression":
        return RegressionFitDiagnostics(
            node=node,
            in_the_money_paths=_required(itm, field="in-the-money path count"),
            observations=_required(observations, field="regression observation count"),
            columns=_required(columns, field="regression column count"),
            rank=_required(rank, field="regression rank"),
            condition_number=_required(condition, field="regression condition"),
            predictor_mean=_required(mean, field="regression predictor mean"),
            predictor_scale=_required(scale, field="regression predictor scale"),
        )
    msg = f"native LSM result returned unsupported diagnostic kind {kind!r}"
    raise LsmError(msg)


def _validate_specs(  # noqa: PLR0913
    *,
    initial_spot: object,
    strike: object,
    schedule: object,
    curve: object,
    dividend_yield_curve: object,
    volatility: object,
    dividend_policy: object,
    executor: object,
    method: object,
) -> None:
    for name, value in (("initial_spot", initial_spot), ("strike", strike)):
        if type(value) is not float:
            msg = f"{name} must be a plain float; observed {type(value).__name__}"
            raise InputError(msg)
    for value, kind, name in (
        (schedule, EventSchedule, "schedule"),
        (curve, LogDiscountCurve, "curve"),
        (dividend_yield_curve, CumulativeDividendYieldCurve, "dividend_yield_curve"),
        (volatility, ConstantVolatility, "volatility"),
        (dividend_policy, DividendPolicy, "dividend_policy"),
    ):
        if type(value) is not kind:
            msg = f"{name} must be {kind.__name__}; observed {type(value).__name__}"
            raise InputError(msg)
    if type(executor) not in (CudaExecutor, CpuExecutor):
        msg = f"executor must be CudaExecutor; observed {type(executor).__name__}"
        raise InputError(msg)
    if type(method) is not Lsm:
        msg = f"method must be Lsm; observed {type(method).__name__}"
        raise InputError(msg)


def price_lsm_call(  # noqa: PLR0913 - financial inputs remain independently typed
    *,
    initial_spot: float,
    strike: float,
    schedule: EventSchedule,
    curve: LogDiscountCurve,
    dividend_yield_curve: CumulativeDividendYieldCurve,
    volatility: ConstantVolatility,
    dividend_policy: DividendPolicy,
    executor: CudaExecutor,
    method: Lsm,
) -> LsmResult:
    """Fit a call stopping policy and evaluate it only on its independent path population.

    Exercise states are observed before any same-node cash dividend. Failures never reduce the
    degree, regularize, reuse training paths, or change the requested executor.

    Raises:
        InputError: If a Python or financial specification is invalid.
        LsmError: If simulation, regression, support, or fixed-policy evaluation fails.
        ExecutionError: If the executor is not a CudaExecutor or the device fails.

    """
    _validate_specs(
        initial_spot=initial_spot,
        strike=strike,
        schedule=schedule,
        curve=curve,
        dividend_yield_curve=dividend_yield_curve,
        volatility=volatility,
        dividend_policy=dividend_policy,
        executor=executor,
        method=method,
    )
    handle = native_executor(executor)
    res = _native.price_lsm_call_seeded_result_f64(
        initial_spot,
        strike,
        list(schedule.times),
        list(curve.times),
        list(curve.log_discounts),
        list(dividend_yield_curve.times),
        list(dividend_yield_curve.cumulative_yields),
        [d.node for d in schedule.dividends],
        [d.amount for d in schedule.dividends],
        list(schedule.exercise_nodes),
        schedule.expiry_node,
        volatility.annualized_decimal,
        dividend_policy.value,
        handle,
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
    price, paths, sd, se, nodes, counts = res.head()
    return LsmResult(
        price=price,
        paths=paths,
        sample_standard_deviation=sd,
        standard_error=se,
        observation_nodes=tuple(nodes),
        exercise_counts=tuple(counts),
        fit_diagnostics=_fit_records(res.rows()),
    )


__all__ = [
    "ExerciseFitDiagnostics",
    "ExerciseTieRule",
    "InsufficientExerciseSupportDiagnostics",
    "InsufficientExerciseSupportPolicy",
    "Lsm",
    "LsmError",
    "LsmResult",
    "NoInTheMoneyPathsDiagnostics",
    "OriginDecisionDiagnostics",
    "RegressionFitDiagnostics",
    "price_lsm_call",
]
