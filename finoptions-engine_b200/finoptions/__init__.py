"""B200-native Longstaff-Schwartz engine with the public API of finoptions' LSM path.

Pricing runs on an explicitly requested ``CudaExecutor`` (one sm_100 device): Philox4x32-10 /
ZIGNOR path simulation, backward stopping-policy fit and independent evaluation are hand-written
CUDA kernels behind the C ABI in include/finoptions_cuda.h. There is no CPU fallback.
"""

from __future__ import annotations

from typing import NamedTuple

from . import _native
from .batch_lsm import (
    BatchDividends,
    CashDividendBatch,
    CashDividendExerciseMesh,
    ContinuousDividendYieldBatch,
    EscrowedCashDividendBatch,
    EscrowedVolatilityConvention,
    ExerciseMesh,
    ExplicitExerciseMesh,
    LsmBatchResult,
    LsmRaggedContracts,
    LsmRaggedGreeks,
    LsmStrikeGroups,
    OriginExercise,
    RaggedExerciseTimes,
    UniformExerciseMesh,
    price_lsm_call_batch,
    price_lsm_call_grouped_batch,
    price_lsm_call_ragged,
    price_lsm_call_ragged_greeks,
    validate_lsm_call_grouped_batch,
    validate_lsm_call_ragged,
)
from .dividends import BatchError, MaturityBoundary, RaggedCashDividends
from .greeks import LsmCallContract, LsmGreeks, lsm_call_price, price_lsm_call_greeks
from .lsm import (
    ExerciseFitDiagnostics,
    ExerciseTieRule,
    InsufficientExerciseSupportDiagnostics,
    InsufficientExerciseSupportPolicy,
    Lsm,
    LsmError,
    LsmResult,
    NoInTheMoneyPathsDiagnostics,
    OriginDecisionDiagnostics,
    RegressionFitDiagnostics,
    price_lsm_call,
)
from .model import (
    CashDividend,
    ConstantVolatility,
    CumulativeDividendYieldCurve,
    DividendPolicy,
    EventSchedule,
    InputError,
    LogDiscountCurve,
)
from .simulation import (
    CpuExecutor,
    CpuMathBackend,
    CudaExecutor,
    DeviceGbmPaths,
    ExecutionError,
    GbmPaths,
    RandomStream,
    SimulationError,
    simulate_gbm,
    simulate_gbm_on_device,
    simulate_gbm_seeded,
)


class BuildInfo(NamedTuple):
    """Native build identity for run manifests."""

    package_version: str
    compiler_version: str


def build_info() -> BuildInfo:
    """Return the loaded engine library's package and compiler identity."""
    return BuildInfo(*_native.build_info())


__version__ = "0.1.0"
__all__ = [
    "BatchDividends",
    "BatchError",
    "BuildInfo",
    "CashDividend",
    "CashDividendBatch",
    "CashDividendExerciseMesh",
    "ConstantVolatility",
    "ContinuousDividendYieldBatch",
    "CpuExecutor",
    "CpuMathBackend",
    "CudaExecutor",
    "CumulativeDividendYieldCurve",
    "DeviceGbmPaths",
    "DividendPolicy",
    "EscrowedCashDividendBatch",
    "EscrowedVolatilityConvention",
    "EventSchedule",
    "ExecutionError",
    "ExerciseFitDiagnostics",
    "ExerciseMesh",
    "ExerciseTieRule",
    "ExplicitExerciseMesh",
    "GbmPaths",
    "InputError",
    "InsufficientExerciseSupportDiagnostics",
    "InsufficientExerciseSupportPolicy",
    "LogDiscountCurve",
    "Lsm",
    "LsmBatchResult",
    "LsmCallContract",
    "LsmError",
    "LsmGreeks",
    "LsmRaggedContracts",
    "LsmRaggedGreeks",
    "LsmResult",
    "LsmStrikeGroups",
    "MaturityBoundary",
    "NoInTheMoneyPathsDiagnostics",
    "OriginDecisionDiagnostics",
    "OriginExercise",
    "RaggedCashDividends",
    "RaggedExerciseTimes",
    "RandomStream",
    "RegressionFitDiagnostics",
    "SimulationError",
    "UniformExerciseMesh",
    "__version__",
    "build_info",
    "lsm_call_price",
    "price_lsm_call",
    "price_lsm_call_batch",
    "price_lsm_call_greeks",
    "price_lsm_call_grouped_batch",
    "price_lsm_call_ragged",
    "price_lsm_call_ragged_greeks",
    "simulate_gbm",
    "simulate_gbm_on_device",
    "simulate_gbm_seeded",
    "validate_lsm_call_grouped_batch",
    "validate_lsm_call_ragged",
]
