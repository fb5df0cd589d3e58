"""GBM simulation from caller normals and the device-resident export, on the device.

The first tests follow the reference's tests/test_simulation.py (adjacent-node transition, the
pre-dividend exercise observation, layout and finiteness checks, input versus simulation errors)
with CudaExecutor in place of CpuExecutor. The rest pin the external-normal route to the oracle and
to the seeded route (the seeded paths' own Philox normals fed back in give the same states, bit for
bit), and check that the device export holds the same values as the host arrays.
"""

from __future__ import annotations

import ctypes
from itertools import pairwise

import _oracle
import numpy as np
import pytest
import torch
from finoptions import (
    CashDividend,
    ConstantVolatility,
    CudaExecutor,
    CumulativeDividendYieldCurve,
    DeviceGbmPaths,
    DividendPolicy,
    EventSchedule,
    InputError,
    LogDiscountCurve,
    RandomStream,
    SimulationError,
    simulate_gbm,
    simulate_gbm_on_device,
    simulate_gbm_seeded,
)
from finoptions import _abi
from finoptions._requests import gbm_seeded_request

pytestmark = pytest.mark.gpu


def inputs(*, dividend: CashDividend | None = None, exercises: tuple[int, ...] = (1, 2)):
    times = (0.0, 0.25, 0.5, 1.0)
    schedule = EventSchedule(times=times, dividends=() if dividend is None else (dividend,),
                             exercise_nodes=exercises, expiry_node=3)
    curve = LogDiscountCurve(times=times, log_discounts=(0.0, -0.01, -0.02, -0.05))
    return schedule, curve, ConstantVolatility(0.20)


def common(schedule, curve, volatility) -> dict:
    return {"initial_spot": 100.0, "schedule": schedule, "curve": curve,
            "dividend_yield_curve": CumulativeDividendYieldCurve.zero(times=schedule.times),
            "volatility": volatility, "dividend_policy": DividendPolicy.LIQUIDATOR, "executor": CudaExecutor()}


def weekly_inputs(dividends=((13, 1.5), (39, 1.5))):
    steps = 52
    times = tuple(i / steps for i in range(steps + 1))
    schedule = EventSchedule(times=times, dividends=tuple(CashDividend(node=n, amount=a) for n, a in dividends),
                             exercise_nodes=tuple(range(1, steps)), expiry_node=steps)
    curve = LogDiscountCurve(times=times, log_discounts=tuple(0.0 if t == 0.0 else -0.04 * t for t in times))
    return schedule, curve, ConstantVolatility(0.25)


def test_matches_the_adjacent_transition_and_time_major_layout() -> None:
    schedule, curve, volatility = inputs()
    normals = np.array([[0.0, 1.0], [0.5, -0.5], [-1.0, 0.25]], dtype=np.float64)
    result = simulate_gbm(**common(schedule, curve, volatility), normals=normals)
    expected = np.empty((3, 2))
    current = np.full(2, 100.0)
    row = 0
    for interval, (left, right) in enumerate(pairwise(schedule.times)):
        variance = volatility.annualized_decimal**2 * (right - left)
        log_drift = -(curve.log_discounts[interval + 1] - curve.log_discounts[interval]) - 0.5 * variance
        current *= np.exp(log_drift + np.sqrt(variance) * normals[interval])
        if interval + 1 in result.observation_nodes:
            expected[row] = current
            row += 1
    assert result.observation_nodes == (1, 2, 3)
    assert result.path_count == 2
    np.testing.assert_allclose(result.states, expected, rtol=2e-15, atol=0.0)
    assert not result.states.flags.writeable
    assert np.shares_memory(result.values_at(1), result.states)


def test_observes_the_pre_dividend_exercise_state() -> None:
    schedule, curve, volatility = inputs(dividend=CashDividend(node=1, amount=200.0), exercises=(1,))
    result = simulate_gbm(**common(schedule, curve, volatility), normals=np.zeros((3, 1)))
    assert result.values_at(1)[0] > 0.0
    assert result.values_at(3)[0] == 0.0


def test_rejects_conversions_and_the_first_non_finite_normal() -> None:
    schedule, curve, volatility = inputs()
    args = common(schedule, curve, volatility)
    with pytest.raises(InputError, match="dtype float64"):
        simulate_gbm(**args, normals=np.zeros((3, 2), dtype=np.float32))
    with pytest.raises(InputError, match="C-contiguous"):
        simulate_gbm(**args, normals=np.zeros((2, 3)).T)
    invalid = np.zeros((3, 2))
    invalid[2, 1] = np.nan
    with pytest.raises(InputError, match="interval 2, path 1: NaN"):
        simulate_gbm(**args, normals=invalid)
    invalid[1, 1] = -np.inf
    with pytest.raises(InputError, match="interval 1, path 1: -inf"):
        simulate_gbm(**args, normals=invalid)


def test_shape_errors_are_input_errors_and_overflow_is_a_simulation_error() -> None:
    schedule, curve, volatility = inputs()
    args = common(schedule, curve, volatility)
    with pytest.raises(InputError, match="normal interval-row buffer length mismatch: expected 3, observed 2"):
        simulate_gbm(**args, normals=np.zeros((2, 2)))
    with pytest.raises(InputError, match="simulation path count must be positive"):
        simulate_gbm(**args, normals=np.zeros((3, 0)))
    overflow = np.zeros((3, 4))
    overflow[0, 2] = 1e308
    overflow[0, 3] = 1e308
    with pytest.raises(SimulationError, match="path 2") as failure:
        simulate_gbm(**args, normals=overflow)
    assert failure.value.path == 2


def _seeded_normals(executor: CudaExecutor, seed: int, domain: int, paths: int, intervals: int) -> np.ndarray:
    """The Philox + ZIGNOR normals path p of the seeded route draws, as [intervals, paths]."""
    per_path = np.zeros(paths * intervals)
    err = _abi.FoError()
    assert _abi.load().fo_sample_standard_normals_f64(
        executor._handle.raw, seed, domain, 0, paths, intervals, per_path.ctypes.data_as(_abi.c_double_p),
        per_path.size, ctypes.byref(err)) == 0, err.message
    return np.ascontiguousarray(per_path.reshape(paths, intervals).T)


def test_the_seeded_paths_own_normals_give_the_seeded_states() -> None:
    schedule, curve, volatility = weekly_inputs()
    args = common(schedule, curve, volatility)
    paths, stream = 20_000, RandomStream(seed=19, domain=4)
    seeded = simulate_gbm_seeded(**args, paths=paths, random_stream=stream)
    normals = _seeded_normals(args["executor"], 19, 4, paths, 52)
    explicit = simulate_gbm(**args, normals=normals)
    assert explicit.observation_nodes == seeded.observation_nodes
    assert np.array_equal(explicit.states.view(np.uint64), seeded.states.view(np.uint64))


@pytest.mark.parametrize("policy", [0, 1])
def test_external_normal_paths_match_the_oracle(policy) -> None:
    schedule, curve, volatility = weekly_inputs(dividends=((13, 1.5), (39, 4.0), (52, 0.5)))
    paths = 30_000
    normals = np.random.default_rng(5).standard_normal((52, paths))
    args = common(schedule, curve, volatility)
    args["dividend_policy"] = DividendPolicy.LIQUIDATOR if policy == 0 else DividendPolicy.SURVIVOR
    gpu = simulate_gbm(**args, normals=normals).states
    req = gbm_seeded_request(
        initial_spot=100.0, schedule_times=schedule.times, curve_times=curve.times, log_discounts=curve.log_discounts,
        dividend_yield_times=schedule.times, cumulative_dividend_yields=[0.0] * len(schedule.times),
        dividend_nodes=[d.node for d in schedule.dividends], dividend_amounts=[d.amount for d in schedule.dividends],
        exercise_nodes=schedule.exercise_nodes, expiry_node=schedule.expiry_node, annualized_volatility=0.25,
        dividend_policy=policy, paths=paths, seed=0, domain=0)
    cpu = _oracle.simulate_from(req, normals)
    # CUDA's exp and glibc's differ in the last bit on some arguments; everything else is exact.
    same = gpu.view(np.uint64) == cpu.view(np.uint64)
    assert same.mean() > 0.5
    assert np.max(np.abs(gpu - cpu) / np.maximum(np.abs(cpu), 1e-300)) <= 1e-13


def test_the_device_export_holds_the_host_values() -> None:
    schedule, curve, volatility = weekly_inputs()
    args = common(schedule, curve, volatility)
    stream = RandomStream(seed=23, domain=6)
    host = simulate_gbm_seeded(**args, paths=50_000, random_stream=stream)
    device = simulate_gbm_on_device(**args, paths=50_000, random_stream=stream)
    assert type(device) is DeviceGbmPaths
    assert device.states.is_cuda and device.states.dtype == torch.float64
    assert tuple(device.states.shape) == host.states.shape and device.path_count == 50_000
    assert np.array_equal(device.states.cpu().numpy().view(np.uint64), host.states.view(np.uint64))
    assert np.array_equal(device.to_host().states, host.states)
    # A DLPack consumer sees the same device memory, without a copy.
    shared = torch.utils.dlpack.from_dlpack(torch.utils.dlpack.to_dlpack(device.states))
    assert shared.data_ptr() == device.states.data_ptr()
    row = device.values_at(26)
    assert row.data_ptr() == device.states[25].data_ptr()


def test_device_normals_give_the_host_normal_states() -> None:
    schedule, curve, volatility = weekly_inputs()
    args = common(schedule, curve, volatility)
    normals = np.random.default_rng(8).standard_normal((52, 40_000))
    host = simulate_gbm(**args, normals=normals)
    device = simulate_gbm_on_device(**args, normals=torch.from_numpy(normals).cuda())
    assert np.array_equal(device.states.cpu().numpy().view(np.uint64), host.states.view(np.uint64))
    bad = torch.from_numpy(normals).cuda()
    bad[7, 123] = float("nan")
    with pytest.raises(InputError, match="interval 7, path 123: NaN"):
        simulate_gbm_on_device(**args, normals=bad)
    with pytest.raises(InputError, match="C-contiguous torch.float64"):
        simulate_gbm_on_device(**args, normals=torch.from_numpy(normals).cuda().T)
    with pytest.raises(InputError, match="either normals or paths"):
        simulate_gbm_on_device(**args, normals=torch.from_numpy(normals).cuda(), paths=10,
                               random_stream=RandomStream(seed=1, domain=1))
