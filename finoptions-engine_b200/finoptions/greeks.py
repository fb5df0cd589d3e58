"""Pathwise adjoint Greeks of the LSM call price with the fitted exercise policy held fixed.

Not in the reference (which obtains sensitivities by bump-and-reprice through price_lsm_call): the
evaluation kernel differentiates every evaluation path in the pass that prices it, so the price
and standard error are exactly those of :func:`finoptions.price_lsm_call` and the Greeks come at
the cost of one evaluation. ``lsm_call_price`` exposes the same computation as a
``torch.autograd.Function`` over the initial spot, the volatility, the log-discount curve and the
cash-dividend amounts.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

from . import _native
from .lsm import Lsm, LsmResult, _fit_diagnostic, _validate_specs
from .model import (
    CashDividend,
    ConstantVolatility,
    CumulativeDividendYieldCurve,
    DividendPolicy,
    EventSchedule,
    LogDiscountCurve,
)
from .simulation import CudaExecutor, native_executor


@dataclass(frozen=True, slots=True)
class LsmGreeks:
    """The priced result and its fixed-policy sensitivities.

    ``log_discount_sensitivities[i]`` is dPrice/dL_i at schedule node i (L the log-discount curve);
    ``dividend_sensitivities[j]`` is dPrice/dD_j for the j-th cash dividend of the schedule.
    """

    result: LsmResult
    delta: float
    vega: float
    log_discount_sensitivities: tuple[float, ...]
    dividend_sensitivities: tuple[float, ...]


def _native_arguments(initial_spot: float, strike: float, schedule: EventSchedule, curve: LogDiscountCurve,
                      dividend_yield_curve: CumulativeDividendYieldCurve, volatility: ConstantVolatility,
                      dividend_policy: DividendPolicy, executor: CudaExecutor, method: Lsm) -> tuple:
    return (
        initial_spot, strike, list(schedule.times), list(curve.times), list(curve.log_discounts),
        list(dividend_yield_curve.times), list(dividend_yield_curve.cumulative_yields),
        [d.node for d in schedule.dividends], [d.amount for d in schedule.dividends], list(schedule.exercise_nodes),
        schedule.expiry_node, volatility.annualized_decimal, dividend_policy.value, native_executor(executor),
        method.training_paths, method.evaluation_paths, method.training_stream.seed, method.training_stream.domain,
        method.evaluation_stream.seed, method.evaluation_stream.domain, method.polynomial_degree,
        method.rank_tolerance, method.condition_limit, method.tie_rule.value,
        method.insufficient_exercise_support.value,
    )


def _result(raw: tuple) -> LsmResult:
    price, paths, sd, se, nodes, counts, diagnostics = raw
    return LsmResult(price=price, paths=paths, sample_standard_deviation=sd, standard_error=se,
                     observation_nodes=tuple(nodes), exercise_counts=tuple(counts),
                     fit_diagnostics=tuple(_fit_diagnostic(d) for d in diagnostics))


def price_lsm_call_greeks(  # noqa: PLR0913 - price_lsm_call's arguments
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
) -> LsmGreeks:
    """Price like :func:`finoptions.price_lsm_call` and return delta, vega and the log-discount and
    cash-dividend sensitivities of the fixed fitted policy's value."""
    _validate_specs(initial_spot=initial_spot, strike=strike, schedule=schedule, curve=curve,
                    dividend_yield_curve=dividend_yield_curve, volatility=volatility,
                    dividend_policy=dividend_policy, executor=executor, method=method)
    raw, delta, vega, d_l, d_d = _native.price_lsm_call_greeks_seeded_f64(
        *_native_arguments(initial_spot, strike, schedule, curve, dividend_yield_curve, volatility, dividend_policy,
                           executor, method))
    return LsmGreeks(result=_result(raw), delta=delta, vega=vega, log_discount_sensitivities=tuple(d_l),
                     dividend_sensitivities=tuple(d_d))


@dataclass(frozen=True, slots=True)
class LsmCallContract:
    """The non-differentiated part of a call priced by :func:`lsm_call_price`: the schedule (times,
    cash-dividend nodes, exercise nodes, expiry), strike, cumulative yields, dividend policy,
    method and executor."""

    strike: float
    times: tuple[float, ...]
    dividend_nodes: tuple[int, ...]
    exercise_nodes: tuple[int, ...]
    expiry_node: int
    cumulative_yields: tuple[float, ...]
    dividend_policy: DividendPolicy
    method: Lsm
    executor: CudaExecutor


def _function() -> Any:
    import torch  # noqa: PLC0415 - torch is only needed by the autograd entry point

    class LsmCallPrice(torch.autograd.Function):
        """Price of an LSM call; backward applies the fixed-policy pathwise adjoint Greeks."""

        @staticmethod
        def forward(ctx: Any, initial_spot: Any, volatility: Any, log_discounts: Any, dividend_amounts: Any,
                    contract: LsmCallContract) -> Any:
            c = contract
            schedule = EventSchedule(
                times=c.times,
                dividends=tuple(CashDividend(node=n, amount=float(a))
                                for n, a in zip(c.dividend_nodes, dividend_amounts.detach().cpu().tolist(), strict=True)),
                exercise_nodes=c.exercise_nodes, expiry_node=c.expiry_node)
            greeks = price_lsm_call_greeks(
                initial_spot=float(initial_spot.detach().cpu()), strike=c.strike, schedule=schedule,
                curve=LogDiscountCurve(times=c.times, log_discounts=tuple(log_discounts.detach().cpu().tolist())),
                dividend_yield_curve=CumulativeDividendYieldCurve(times=c.times, cumulative_yields=c.cumulative_yields),
                volatility=ConstantVolatility(float(volatility.detach().cpu())), dividend_policy=c.dividend_policy,
                executor=c.executor, method=c.method)
            f64 = {"dtype": torch.float64, "device": initial_spot.device}
            ctx.save_for_backward(torch.tensor(greeks.delta, **f64), torch.tensor(greeks.vega, **f64),
                                  torch.tensor(greeks.log_discount_sensitivities, **f64),
                                  torch.tensor(greeks.dividend_sensitivities, **f64))
            return torch.tensor(greeks.result.price, **f64)

        @staticmethod
        def backward(ctx: Any, grad: Any) -> tuple:
            delta, vega, d_l, d_d = ctx.saved_tensors
            return grad * delta, grad * vega, grad * d_l, grad * d_d, None

    return LsmCallPrice


_LSM_CALL_PRICE: Any = None


def lsm_call_price(initial_spot: Any, volatility: Any, log_discounts: Any, dividend_amounts: Any,
                   contract: LsmCallContract) -> Any:
    """Differentiable LSM call price (a float64 scalar tensor).

    ``initial_spot`` and ``volatility`` are scalar tensors, ``log_discounts`` has one entry per
    schedule node and ``dividend_amounts`` one per cash dividend. ``backward`` returns delta, vega
    and the log-discount and dividend sensitivities of the fixed fitted policy (common random
    numbers: the same Philox streams as the forward price)."""
    global _LSM_CALL_PRICE  # noqa: PLW0603 - the autograd class is built once, on first use
    if _LSM_CALL_PRICE is None:
        _LSM_CALL_PRICE = _function()
    return _LSM_CALL_PRICE.apply(initial_spot, volatility, log_discounts, dividend_amounts, contract)


__all__ = ["LsmCallContract", "LsmGreeks", "lsm_call_price", "price_lsm_call_greeks"]
