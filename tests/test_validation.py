"""Host-side validation: the reference's typed errors and messages, without a device."""

from __future__ import annotations

import ctypes
from typing import cast

import numpy as np
import pytest
from finoptions import (
    CashDividend,
    ConstantVolatility,
    CpuExecutor,
    CudaExecutor,
    CumulativeDividendYieldCurve,
    EventSchedule,
    ExerciseTieRule,
    InputError,
    InsufficientExerciseSupportPolicy,
    LogDiscountCurve,
    Lsm,
    RaggedCashDividends,
    RaggedExerciseTimes,
    RandomStream,
    UniformExerciseMesh,
    OriginExercise,
    BatchError,
)
from finoptions import _abi
from finoptions._requests import lsm_call_request


def method(**kw):
    base = dict(training_paths=100, evaluation_paths=100, training_stream=RandomStream(seed=1, domain=1),
                evaluation_stream=RandomStream(seed=1, domain=2),
                insufficient_exercise_support=InsufficientExerciseSupportPolicy.FAIL)
    base.update(kw)
    return Lsm(**base)


def test_lsm_configuration_fails_instead_of_substituting() -> None:
    with pytest.raises(InputError, match="training_paths must be a plain int"):
        method(training_paths=cast("int", True))
    with pytest.raises(InputError, match="different domains"):
        method(evaluation_stream=RandomStream(seed=2, domain=1))
    with pytest.raises(InputError, match="polynomial_degree"):
        method(polynomial_degree=5)
    with pytest.raises(InputError, match="tie_rule must be ExerciseTieRule"):
        method(tie_rule=cast("ExerciseTieRule", "strictly_greater"))
    with pytest.raises(InputError, match="insufficient_exercise_support"):
        method(insufficient_exercise_support=cast("InsufficientExerciseSupportPolicy", "continue"))
    with pytest.raises(InputError, match="condition_limit"):
        method(rank_tolerance=1e-3, condition_limit=1e8)


def test_schedule_and_curve_messages_match_the_reference() -> None:
    with pytest.raises(InputError, match="time grid must be strictly increasing; node 1 is 0.5 and node 2 is 0.5"):
        EventSchedule(times=(0.0, 0.5, 0.5), dividends=(), exercise_nodes=(), expiry_node=2)
    with pytest.raises(InputError, match="time grid must begin at exactly 0.0; observed 0.1"):
        EventSchedule(times=(0.1, 0.5), dividends=(), exercise_nodes=(), expiry_node=1)
    with pytest.raises(InputError, match="expiry must be the final non-origin node 2; observed node 1"):
        EventSchedule(times=(0.0, 0.5, 1.0), dividends=(), exercise_nodes=(), expiry_node=1)
    with pytest.raises(InputError, match="exercise opportunity at node 2 must occur before expiry node 2"):
        EventSchedule(times=(0.0, 0.5, 1.0), dividends=(), exercise_nodes=(2,), expiry_node=2)
    with pytest.raises(InputError, match="cash dividend at node 0 must occur strictly after valuation"):
        EventSchedule(times=(0.0, 1.0), dividends=(CashDividend(node=0, amount=1.0),), exercise_nodes=(), expiry_node=1)
    with pytest.raises(InputError, match="cash-dividend schedule repeats node 1"):
        EventSchedule(times=(0.0, 0.5, 1.0), dividends=(CashDividend(node=1, amount=1.0), CashDividend(node=1, amount=2.0)),
                      exercise_nodes=(), expiry_node=2)
    with pytest.raises(InputError, match="node 3 is outside a time grid containing 3 nodes"):
        EventSchedule(times=(0.0, 0.5, 1.0), dividends=(), exercise_nodes=(3,), expiry_node=2)
    with pytest.raises(InputError, match="log discount at node 0 must be exactly 0.0"):
        LogDiscountCurve(times=(0.0, 1.0), log_discounts=(0.001, -0.01))
    with pytest.raises(InputError, match="log-discount curve has 1 nodes; time grid requires 2"):
        LogDiscountCurve(times=(0.0, 1.0), log_discounts=(0.0,))
    with pytest.raises(InputError, match="cumulative dividend yield must be nondecreasing"):
        CumulativeDividendYieldCurve(times=(0.0, 0.5, 1.0), cumulative_yields=(0.0, 0.02, 0.01))
    with pytest.raises(InputError, match="constant annualized volatility must be finite and strictly positive; observed 0.0"):
        ConstantVolatility(0.0)
    with pytest.raises(InputError, match="observed -1.0"):
        CashDividend(node=1, amount=-1.0)
    with pytest.raises(InputError, match="observed NaN"):
        CashDividend(node=1, amount=float("nan"))


def test_float_rendering_follows_rust_debug() -> None:
    for value, text in ((1e-5, "1e-5"), (100.0, "100.0"), (0.1, "0.1"), (1.5e20, "1.5e20"), (-0.0, "-0.0"),
                        (float("inf"), "inf"), (1e16, "1e16"), (123456.789, "123456.789")):
        with pytest.raises(InputError) as failure:
            LogDiscountCurve(times=(0.0, 1.0), log_discounts=(value, 0.0))
        if value == 0.0:
            continue
        assert str(failure.value).endswith(text), (value, str(failure.value))


def test_ragged_buffers_are_validated_with_batch_errors() -> None:
    with pytest.raises(BatchError, match="ragged offsets must contain at least two values; observed 1"):
        RaggedCashDividends(offsets=np.array([0], dtype=np.int64), times=np.zeros(0), amounts=np.zeros(0))
    with pytest.raises(BatchError, match="cash-dividend times must be nondecreasing"):
        RaggedCashDividends(offsets=np.array([0, 2], dtype=np.int64), times=np.array([0.2, 0.1]), amounts=np.ones(2))
    with pytest.raises(BatchError, match="exercise times must be strictly increasing"):
        RaggedExerciseTimes(offsets=np.array([0, 2], dtype=np.int64), times=np.array([0.2, 0.2]))
    with pytest.raises(BatchError, match="ragged offset span"):
        RaggedExerciseTimes(offsets=np.array([0, 3], dtype=np.int64), times=np.array([0.2, 0.3]))
    sliced = RaggedCashDividends(offsets=np.array([2, 3, 5], dtype=np.int64), times=np.array([0.1, 0.2, 0.3]),
                                 amounts=np.ones(3))
    assert sliced.rows == 2


def test_uniform_mesh_requires_explicit_origin() -> None:
    with pytest.raises(InputError, match="base_intervals"):
        UniformExerciseMesh(base_intervals=0, origin_exercise=OriginExercise.EXCLUDED)
    with pytest.raises(InputError, match="origin_exercise"):
        UniformExerciseMesh(base_intervals=4, origin_exercise=cast("OriginExercise", "excluded"))


def native_request(**overrides):
    base = dict(
        initial_spot=100.0, strike=100.0, schedule_times=[0.0, 0.5, 1.0], curve_times=[0.0, 0.5, 1.0],
        log_discounts=[0.0, -0.01, -0.025], dividend_yield_times=[0.0, 0.5, 1.0],
        cumulative_dividend_yields=[0.0, 0.0, 0.0], dividend_nodes=[1], dividend_amounts=[2.0], exercise_nodes=[1],
        expiry_node=2, annualized_volatility=0.2, dividend_policy=0, training_paths=4096, evaluation_paths=4096,
        training_seed=7, training_domain=1, evaluation_seed=7, evaluation_domain=2, polynomial_degree=4,
        rank_tolerance=1e-12, condition_limit=1e8, tie_rule=0, insufficient_exercise_support=0,
    )
    base.update(overrides)
    return lsm_call_request(**base)


def validate(request) -> tuple[int, int, str]:
    lib = _abi.load()
    lib.fo_validate_lsm_call_request.argtypes = [ctypes.POINTER(_abi.FoLsmCallRequest), ctypes.POINTER(_abi.FoError)]
    err = _abi.FoError()
    status = lib.fo_validate_lsm_call_request(ctypes.byref(request.struct), ctypes.byref(err))
    return status, err.code, err.message.decode()


def test_single_contract_request_validation_order_and_messages() -> None:
    assert validate(native_request())[0] == 0
    status, _, message = validate(native_request(curve_times=[0.0, 0.25, 1.0]))
    assert status == _abi.FO_ERR_SIMULATION and message == "discount curve and event schedule must use the identical time grid"
    status, _, message = validate(native_request(polynomial_degree=5))
    assert status == _abi.FO_ERR_LSM and "the validated maximum degree is 4" in message
    status, _, message = validate(native_request(training_domain=2))
    assert status == _abi.FO_ERR_LSM and "both use domain 2" in message
    status, _, message = validate(native_request(strike=-1.0))
    assert status == _abi.FO_ERR_LSM and message == "call strike must be finite and strictly positive; observed -1.0"
    status, _, message = validate(native_request(initial_spot=float("nan")))
    assert status == _abi.FO_ERR_LSM and message.startswith("LSM training simulation failed: initial spot")
    status, _, message = validate(native_request(training_paths=0))
    assert message == "LSM training simulation failed: simulation path count must be positive"
    status, _, message = validate(native_request(dividend_policy=7))
    assert status == _abi.FO_ERR_INPUT and message.startswith("unsupported dividend policy")


def test_cpu_executor_is_not_a_fallback() -> None:
    from finoptions import ExecutionError, price_lsm_call
    from finoptions.model import DividendPolicy

    schedule = EventSchedule(times=(0.0, 1.0), dividends=(), exercise_nodes=(), expiry_node=1)
    with pytest.raises(ExecutionError, match="prices only on CudaExecutor"):
        price_lsm_call(
            initial_spot=100.0, strike=100.0, schedule=schedule,
            curve=LogDiscountCurve(times=schedule.times, log_discounts=(0.0, -0.05)),
            dividend_yield_curve=CumulativeDividendYieldCurve.zero(times=schedule.times),
            volatility=ConstantVolatility(0.2), dividend_policy=DividendPolicy.LIQUIDATOR,
            executor=CpuExecutor(threads=2), method=method(),
        )
    assert CudaExecutor is not CpuExecutor


def test_simulation_entries_do_not_fall_back_to_the_cpu() -> None:
    from finoptions import ExecutionError, simulate_gbm, simulate_gbm_on_device
    from finoptions.model import DividendPolicy

    schedule = EventSchedule(times=(0.0, 0.5, 1.0), dividends=(), exercise_nodes=(1,), expiry_node=2)
    common = dict(initial_spot=100.0, schedule=schedule,
                  curve=LogDiscountCurve(times=schedule.times, log_discounts=(0.0, -0.02, -0.05)),
                  dividend_yield_curve=CumulativeDividendYieldCurve.zero(times=schedule.times),
                  volatility=ConstantVolatility(0.2), dividend_policy=DividendPolicy.LIQUIDATOR,
                  executor=CpuExecutor(threads=2))
    with pytest.raises(ExecutionError, match="prices only on CudaExecutor"):
        simulate_gbm(**common, normals=np.zeros((2, 4)))
    with pytest.raises(ExecutionError, match="prices only on CudaExecutor"):
        simulate_gbm_on_device(**common, paths=4, random_stream=RandomStream(seed=1, domain=1))
    with pytest.raises(InputError, match="initial_spot must be a plain float"):
        simulate_gbm(**{**common, "initial_spot": 100}, normals=np.zeros((2, 4)))
