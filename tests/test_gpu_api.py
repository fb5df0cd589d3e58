"""Public-API tests on the device, following the reference's tests/test_lsm.py and
tests/test_simulation.py, with CudaExecutor in place of CpuExecutor."""

from __future__ import annotations

from math import erfc, exp, log, sqrt

import numpy as np
import pytest
from finoptions import (
    CashDividend,
    ConstantVolatility,
    CudaExecutor,
    CumulativeDividendYieldCurve,
    DividendPolicy,
    EventSchedule,
    ExerciseTieRule,
    InsufficientExerciseSupportDiagnostics,
    InsufficientExerciseSupportPolicy,
    LogDiscountCurve,
    Lsm,
    LsmError,
    OriginDecisionDiagnostics,
    RandomStream,
    RegressionFitDiagnostics,
    price_lsm_call,
    simulate_gbm_seeded,
)

pytestmark = pytest.mark.gpu


def one_dividend_inputs():
    schedule = EventSchedule(times=(0.0, 0.5, 1.0), dividends=(CashDividend(node=1, amount=7.0),),
                             exercise_nodes=(1,), expiry_node=2)
    curve = LogDiscountCurve(times=schedule.times, log_discounts=(0.0, -0.03, -0.06))
    return schedule, curve, ConstantVolatility(0.30)


def method(paths: int = 32768, support=InsufficientExerciseSupportPolicy.FAIL) -> Lsm:
    return Lsm(training_paths=paths, evaluation_paths=paths, training_stream=RandomStream(seed=10_000, domain=1),
               evaluation_stream=RandomStream(seed=20_000, domain=2), insufficient_exercise_support=support,
               polynomial_degree=4, rank_tolerance=1.0e-12, condition_limit=1.0e8,
               tie_rule=ExerciseTieRule.STRICTLY_GREATER)


def test_public_lsm_is_deterministic_and_returns_complete_diagnostics() -> None:
    schedule, curve, volatility = one_dividend_inputs()
    common = dict(initial_spot=100.0, strike=100.0, schedule=schedule, curve=curve,
                  dividend_yield_curve=CumulativeDividendYieldCurve.zero(times=schedule.times),
                  volatility=volatility, dividend_policy=DividendPolicy.LIQUIDATOR, method=method())
    first = price_lsm_call(**common, executor=CudaExecutor(device=0))
    second = price_lsm_call(**common, executor=CudaExecutor(device=0))
    assert first == second
    assert first.observation_nodes == (1, 2)
    assert sum(first.exercise_counts) == first.paths == 32768
    assert len(first.fit_diagnostics) == 1
    regression = first.fit_diagnostics[0]
    assert isinstance(regression, RegressionFitDiagnostics)
    assert regression.observations == regression.in_the_money_paths
    assert regression.columns == regression.rank == 5
    assert regression.condition_number < 1.0e8


def test_origin_exercise_is_reported_as_one_common_decision() -> None:
    schedule = EventSchedule(times=(0.0, 0.5, 1.0), dividends=(CashDividend(node=1, amount=200.0),),
                             exercise_nodes=(0,), expiry_node=2)
    result = price_lsm_call(
        initial_spot=200.0, strike=100.0, schedule=schedule,
        curve=LogDiscountCurve(times=schedule.times, log_discounts=(0.0, 0.0, 0.0)),
        dividend_yield_curve=CumulativeDividendYieldCurve.zero(times=schedule.times),
        volatility=ConstantVolatility(0.30), dividend_policy=DividendPolicy.LIQUIDATOR,
        executor=CudaExecutor(), method=method(paths=1_000),
    )
    assert result.price == 100.0
    assert result.exercise_counts == (1_000, 0)
    assert isinstance(result.fit_diagnostics[0], OriginDecisionDiagnostics)
    assert result.fit_diagnostics[0].exercise


def test_continuous_yield_european_slice_covers_black_scholes_merton() -> None:
    spot, strike, rate, q, sigma, maturity = 100.0, 105.0, 0.05, 0.02, 0.25, 1.25
    schedule = EventSchedule(times=(0.0, maturity), dividends=(), exercise_nodes=(), expiry_node=1)
    result = price_lsm_call(
        initial_spot=spot, strike=strike, schedule=schedule,
        curve=LogDiscountCurve(times=schedule.times, log_discounts=(0.0, -rate * maturity)),
        dividend_yield_curve=CumulativeDividendYieldCurve.constant(times=schedule.times, annualized_decimal=q),
        volatility=ConstantVolatility(sigma), dividend_policy=DividendPolicy.LIQUIDATOR,
        executor=CudaExecutor(), method=method(paths=131_072),
    )
    srt = sigma * sqrt(maturity)
    d1 = (log(spot / strike) + (rate - q + 0.5 * sigma**2) * maturity) / srt
    cdf = lambda x: 0.5 * erfc(-x / sqrt(2.0))  # noqa: E731
    expected = spot * exp(-q * maturity) * cdf(d1) - strike * exp(-rate * maturity) * cdf(d1 - srt)
    assert result.standard_error is not None
    assert abs(result.price - expected) <= 5.0 * result.standard_error
    assert result.fit_diagnostics == ()


def test_insufficient_support_fails_or_continues_as_declared() -> None:
    schedule, curve, volatility = one_dividend_inputs()
    common = dict(initial_spot=100.0, strike=100.0, schedule=schedule, curve=curve,
                  dividend_yield_curve=CumulativeDividendYieldCurve.zero(times=schedule.times),
                  volatility=volatility, dividend_policy=DividendPolicy.LIQUIDATOR, executor=CudaExecutor())
    with pytest.raises(LsmError, match="requires at least 5"):
        price_lsm_call(**common, method=method(paths=4))
    result = price_lsm_call(**common, method=method(paths=4, support=InsufficientExerciseSupportPolicy.CONTINUE))
    assert result.exercise_counts == (0, 4)
    assert result.fit_diagnostics == (
        InsufficientExerciseSupportDiagnostics(node=1, in_the_money_paths=3, required_paths=5),
    )


def test_seeded_simulation_moments_and_terminal_mean() -> None:
    steps = 12
    times = tuple(i / steps for i in range(steps + 1))
    schedule = EventSchedule(times=times, dividends=(), exercise_nodes=tuple(range(1, steps)), expiry_node=steps)
    paths = simulate_gbm_seeded(
        initial_spot=100.0, schedule=schedule,
        curve=LogDiscountCurve(times=times, log_discounts=tuple(0.0 if t == 0.0 else -0.03 * t for t in times)),
        dividend_yield_curve=CumulativeDividendYieldCurve.zero(times=times), volatility=ConstantVolatility(0.2),
        dividend_policy=DividendPolicy.LIQUIDATOR, executor=CudaExecutor(), paths=200_000,
        random_stream=RandomStream(seed=3, domain=9),
    )
    assert paths.states.shape == (steps, 200_000)
    assert not paths.states.flags.writeable
    terminal = paths.values_at(steps)
    assert abs(terminal.mean() - 100.0 * exp(0.03)) < 5 * terminal.std() / sqrt(terminal.size)
    log_returns = np.log(paths.states[1] / paths.states[0])
    assert abs(log_returns.std() - 0.2 * sqrt(1 / steps)) < 0.002
