"""Executors, random streams and seeded GBM path simulation.

``CudaExecutor`` is the engine's execution resource: one B200 device, requested explicitly,
failing at construction when none is present. ``CpuExecutor`` keeps the reference's value type
(python/finoptions/simulation.py:40-62) so request code ports unchanged, but this engine has no CPU
pricing path: passing it to a pricing function raises ``ExecutionError`` instead of falling back.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from enum import StrEnum
from itertools import pairwise
from typing import Any, Final

import numpy as np
import numpy.typing as npt

from . import _native
from .model import (
    ConstantVolatility,
    CumulativeDividendYieldCurve,
    DividendPolicy,
    EventSchedule,
    InputError,
    LogDiscountCurve,
)

Float64Matrix = npt.NDArray[np.float64]
ExecutionError = _native.ExecutionError
SimulationError = _native.SimulationError
_MAX_SEED: Final = (2**64) - 1
_MAX_DOMAIN: Final = (2**32) - 1
_MAX_PATHS: Final = (2**32) - 1


class CpuMathBackend(StrEnum):
    """Named floating-point implementation of the reference's CPU kernels."""

    RUST_STD_F64 = "rust_std_f64"
    APPLE_ACCELERATE = "apple_accelerate"


@dataclass(frozen=True, slots=True)
class CpuExecutor:
    """The reference's CPU resource description. The B200 engine does not execute on it."""

    threads: int
    math_backend: CpuMathBackend = CpuMathBackend.RUST_STD_F64

    def __post_init__(self) -> None:
        """Reject inferred or empty thread counts like the reference."""
        if type(self.threads) is not int or self.threads <= 0:
            msg = f"threads must be a positive plain int; observed {self.threads!r}"
            raise InputError(msg)
        if type(self.math_backend) is not CpuMathBackend:
            msg = f"math_backend must be CpuMathBackend; observed {type(self.math_backend).__name__}"
            raise InputError(msg)


_EXECUTORS: dict[int, _native.CudaExecutor] = {}


@dataclass(frozen=True, slots=True)
class CudaExecutor:
    """One explicitly requested sm_100 (B200) device. There is no CPU fallback.

    Executors of the same device share one native executor (stream + device arena) per process.
    """

    device: int = 0
    _handle: _native.CudaExecutor = field(init=False, repr=False, compare=False)

    def __post_init__(self) -> None:
        """Open the device once and fail fast when it is absent or not a Blackwell part."""
        if type(self.device) is not int or self.device < 0:
            msg = f"device must be a nonnegative plain int; observed {self.device!r}"
            raise InputError(msg)
        handle = _EXECUTORS.get(self.device)
        if handle is None:
            handle = _native.CudaExecutor(self.device)
            _EXECUTORS[self.device] = handle
        object.__setattr__(self, "_handle", handle)


def native_executor(executor: object) -> _native.CudaExecutor:
    """Return the native handle of a CudaExecutor, or fail without falling back."""
    if type(executor) is CudaExecutor:
        return executor._handle  # noqa: SLF001 - package-private handle
    if type(executor) is CpuExecutor:
        msg = "CpuExecutor selects the reference CPU engine; the B200 engine prices only on CudaExecutor"
        raise ExecutionError(msg)
    msg = f"executor must be CudaExecutor; observed {type(executor).__name__}"
    raise InputError(msg)


@dataclass(frozen=True, slots=True)
class RandomStream:
    """Reproducible Philox namespace (seed, domain) for one statistically distinct path set."""

    seed: int
    domain: int

    def __post_init__(self) -> None:
        """Reject signs, booleans and values outside the counter layout."""
        if type(self.seed) is not int or not 0 <= self.seed <= _MAX_SEED:
            msg = f"seed must be a plain int in [0, {_MAX_SEED}]; observed {self.seed!r}"
            raise InputError(msg)
        if type(self.domain) is not int or not 0 <= self.domain <= _MAX_DOMAIN:
            msg = f"domain must be a plain int in [0, {_MAX_DOMAIN}]; observed {self.domain!r}"
            raise InputError(msg)


@dataclass(frozen=True, slots=True)
class GbmPaths:
    """Time-major pre-event states at exercise nodes followed by the post-event expiry state."""

    observation_nodes: tuple[int, ...]
    states: Float64Matrix

    def __post_init__(self) -> None:
        """Check the native output contract."""
        if (
            type(self.observation_nodes) is not tuple
            or not self.observation_nodes
            or any(type(node) is not int or node < 0 or node > _MAX_DOMAIN for node in self.observation_nodes)
        ):
            msg = "observation_nodes must be an immutable tuple[int, ...]"
            raise InputError(msg)
        if any(right <= left for left, right in pairwise(self.observation_nodes)):
            msg = "observation_nodes must be strictly increasing"
            raise InputError(msg)
        if type(self.states) is not np.ndarray or self.states.dtype != np.dtype(np.float64):
            msg = "states must be a float64 numpy.ndarray"
            raise InputError(msg)
        if self.states.ndim != 2 or self.states.shape[0] != len(self.observation_nodes):  # noqa: PLR2004
            msg = f"states must have shape [observation_nodes, paths]; observed {self.states.shape!r}"
            raise InputError(msg)
        if self.states.shape[1] == 0:
            msg = "states must contain at least one path"
            raise InputError(msg)

    @property
    def path_count(self) -> int:
        """Number of simulated paths."""
        return self.states.shape[1]

    def values_at(self, node: int) -> npt.NDArray[np.float64]:
        """Zero-copy path row of an observed node."""
        if type(node) is not int:
            msg = f"observation node must be a plain int; observed {type(node).__name__}"
            raise InputError(msg)
        try:
            row = self.observation_nodes.index(node)
        except ValueError as error:
            raise KeyError(node) from error
        return self.states[row]


def _validate_specs(schedule: object, curve: object, dividend_yield_curve: object, volatility: object,
                    dividend_policy: object) -> None:
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


def _plan_arguments(initial_spot: float, schedule: EventSchedule, curve: LogDiscountCurve,
                    dividend_yield_curve: CumulativeDividendYieldCurve, volatility: ConstantVolatility,
                    dividend_policy: DividendPolicy) -> tuple:
    return (
        initial_spot,
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
    )


def _validate_normal_matrix(normals: object) -> None:
    # _validate_normal_matrix (python/finoptions/simulation.py:181-193): borrowed, never cast or copied.
    if type(normals) is not np.ndarray:
        msg = f"normals must be a plain numpy.ndarray; observed {type(normals).__name__}"
        raise InputError(msg)
    if normals.dtype != np.dtype(np.float64):
        msg = f"normals must have dtype float64; observed {normals.dtype}"
        raise InputError(msg)
    if normals.ndim != 2:  # noqa: PLR2004 - [intervals, paths]
        msg = f"normals must have shape [intervals, paths]; observed {normals.shape!r}"
        raise InputError(msg)
    if not normals.flags.c_contiguous:
        msg = "normals must be C-contiguous; implicit copies are forbidden"
        raise InputError(msg)


def simulate_gbm(  # noqa: PLR0913 - each financial input is independently typed
    *,
    initial_spot: float,
    schedule: EventSchedule,
    curve: LogDiscountCurve,
    dividend_yield_curve: CumulativeDividendYieldCurve,
    volatility: ConstantVolatility,
    dividend_policy: DividendPolicy,
    executor: CudaExecutor,
    normals: Float64Matrix,
) -> GbmPaths:
    """Simulate exact adjacent-node GBM paths on the device from explicit standard normals
    (simulate_gbm, python/finoptions/simulation.py:210-259).

    ``normals`` is a C-contiguous float64 matrix [intervals, paths], read without casting or
    copying on the host. Every variate is checked for finiteness before any path is computed.

    Raises:
        InputError: If a runtime type, grid, shape, value, or financial input is invalid.
        SimulationError: For a wrong interval-row count, an empty path set, a non-finite variate or
            a non-finite path transition.

    """
    if type(initial_spot) is not float:
        msg = f"initial_spot must be a plain float; observed {type(initial_spot).__name__}"
        raise InputError(msg)
    _validate_specs(schedule, curve, dividend_yield_curve, volatility, dividend_policy)
    handle = native_executor(executor)
    _validate_normal_matrix(normals)
    states = _native.simulate_gbm_f64(
        *_plan_arguments(initial_spot, schedule, curve, dividend_yield_curve, volatility, dividend_policy),
        handle,
        normals,
    )
    states.flags.writeable = False
    return GbmPaths(observation_nodes=(*schedule.exercise_nodes, schedule.expiry_node), states=states)


@dataclass(frozen=True, slots=True)
class DeviceGbmPaths:
    """GbmPaths whose states stay in device memory: a torch.float64 tensor [observations, paths] on
    the executor's device, time-major like GbmPaths.states. ``to_host()`` copies it to GbmPaths."""

    observation_nodes: tuple[int, ...]
    states: Any

    @property
    def path_count(self) -> int:
        """Number of simulated paths."""
        return int(self.states.shape[1])

    def values_at(self, node: int) -> Any:
        """The device row of an observed node (a view, no copy)."""
        if type(node) is not int:
            msg = f"observation node must be a plain int; observed {type(node).__name__}"
            raise InputError(msg)
        try:
            row = self.observation_nodes.index(node)
        except ValueError as error:
            raise KeyError(node) from error
        return self.states[row]

    def to_host(self) -> GbmPaths:
        """Copy the states to host memory as read-only GbmPaths."""
        states = self.states.cpu().numpy()
        states.flags.writeable = False
        return GbmPaths(observation_nodes=self.observation_nodes, states=states)


def simulate_gbm_on_device(  # noqa: PLR0913 - each financial input is independently typed
    *,
    initial_spot: float,
    schedule: EventSchedule,
    curve: LogDiscountCurve,
    dividend_yield_curve: CumulativeDividendYieldCurve,
    volatility: ConstantVolatility,
    dividend_policy: DividendPolicy,
    executor: CudaExecutor,
    paths: int | None = None,
    random_stream: RandomStream | None = None,
    normals: Any = None,
) -> DeviceGbmPaths:
    """simulate_gbm_seeded or simulate_gbm with the states left on the device.

    Give either ``paths`` and ``random_stream`` (Philox streams, the same values as
    simulate_gbm_seeded) or ``normals``, a C-contiguous torch.float64 tensor [intervals, paths] on
    the executor's device (the same values as simulate_gbm on those normals). The returned tensor
    is written by the kernel in place; nothing passes through host memory. For further device work
    (a caller's own regression, a DLPack consumer) without a host round trip.
    """
    if type(initial_spot) is not float:
        msg = f"initial_spot must be a plain float; observed {type(initial_spot).__name__}"
        raise InputError(msg)
    _validate_specs(schedule, curve, dividend_yield_curve, volatility, dividend_policy)
    handle = native_executor(executor)
    if normals is None:
        if type(paths) is not int or not 1 <= paths <= _MAX_PATHS:
            msg = f"paths must be a plain int in [1, {_MAX_PATHS}]; observed {paths!r}"
            raise InputError(msg)
        if type(random_stream) is not RandomStream:
            msg = f"random_stream must be RandomStream; observed {type(random_stream).__name__}"
            raise InputError(msg)
        seed, domain = random_stream.seed, random_stream.domain
    else:
        if paths is not None or random_stream is not None:
            msg = "give either normals or paths with a random_stream, not both"
            raise InputError(msg)
        seed, domain, paths = 0, 0, 0
    states = _native.simulate_gbm_device_f64(
        *_plan_arguments(initial_spot, schedule, curve, dividend_yield_curve, volatility, dividend_policy),
        handle,
        paths,
        seed,
        domain,
        normals,
    )
    return DeviceGbmPaths(observation_nodes=(*schedule.exercise_nodes, schedule.expiry_node), states=states)


def simulate_gbm_seeded(  # noqa: PLR0913 - each financial input is independently typed
    *,
    initial_spot: float,
    schedule: EventSchedule,
    curve: LogDiscountCurve,
    dividend_yield_curve: CumulativeDividendYieldCurve,
    volatility: ConstantVolatility,
    dividend_policy: DividendPolicy,
    executor: CudaExecutor,
    paths: int,
    random_stream: RandomStream,
) -> GbmPaths:
    """Generate and evolve reproducible GBM paths on the device (Philox4x32-10 + ZIGNOR).

    Path i is a pure function of (seed, domain, i). Returns only the pre-event exercise states and
    the terminal expiry state, time-major.
    """
    if type(initial_spot) is not float:
        msg = f"initial_spot must be a plain float; observed {type(initial_spot).__name__}"
        raise InputError(msg)
    _validate_specs(schedule, curve, dividend_yield_curve, volatility, dividend_policy)
    handle = native_executor(executor)
    if type(paths) is not int or not 1 <= paths <= _MAX_PATHS:
        msg = f"paths must be a plain int in [1, {_MAX_PATHS}]; observed {paths!r}"
        raise InputError(msg)
    if type(random_stream) is not RandomStream:
        msg = f"random_stream must be RandomStream; observed {type(random_stream).__name__}"
        raise InputError(msg)
    states = _native.simulate_gbm_seeded_f64(
        *_plan_arguments(initial_spot, schedule, curve, dividend_yield_curve, volatility, dividend_policy),
        handle,
        paths,
        random_stream.seed,
        random_stream.domain,
    )
    states.flags.writeable = False
    return GbmPaths(observation_nodes=(*schedule.exercise_nodes, schedule.expiry_node), states=states)


__all__ = [
    "CpuExecutor",
    "CpuMathBackend",
    "CudaExecutor",
    "DeviceGbmPaths",
    "ExecutionError",
    "GbmPaths",
    "RandomStream",
    "SimulationError",
    "native_executor",
    "simulate_gbm",
    "simulate_gbm_on_device",
    "simulate_gbm_seeded",
]
