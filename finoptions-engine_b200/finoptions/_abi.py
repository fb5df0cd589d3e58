"""ctypes image of include/finoptions_cuda.h and the loader of the engine's shared library.

The shared library is built in-tree (``finoptions-engine_b200/finoptions/_lib/``) by
``finoptions-engine_b200/build.py``. There is no fallback: if the library is absent, importing a
pricing entry point raises ``ExecutionError`` naming the missing file.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Final

c_double_p = ctypes.POINTER(ctypes.c_double)
c_uint32_p = ctypes.POINTER(ctypes.c_uint32)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)

FO_OK: Final = 0
FO_ERR_INPUT: Final = 1
FO_ERR_LSM: Final = 2
FO_ERR_SIMULATION: Final = 3
FO_ERR_EXECUTION: Final = 4
FO_ERR_BATCH: Final = 5

FO_DIAG_ORIGIN_DECISION: Final = 0
FO_DIAG_NO_IN_THE_MONEY_PATHS: Final = 1
FO_DIAG_INSUFFICIENT_SUPPORT: Final = 2
FO_DIAG_REGRESSION: Final = 3

ERROR_MESSAGE_CAPACITY: Final = 1024


class FoError(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("code", ctypes.c_int32),
        ("row", ctypes.c_int64),
        ("group", ctypes.c_int64),
        ("node", ctypes.c_int64),
        ("path", ctypes.c_int64),
        ("message", ctypes.c_char * ERROR_MESSAGE_CAPACITY),
    ]


class FoLsmCallRequest(ctypes.Structure):
    # The single-contract call is latency-bound on the host: its array fields take plain addresses
    # (set from integers) into buffers that the request object keeps alive.
    _fields_ = [
        ("initial_spot", ctypes.c_double),
        ("strike", ctypes.c_double),
        ("schedule_times", ctypes.c_void_p), ("n_schedule_times", ctypes.c_uint64),
        ("curve_times", ctypes.c_void_p), ("n_curve_times", ctypes.c_uint64),
        ("log_discounts", ctypes.c_void_p), ("n_log_discounts", ctypes.c_uint64),
        ("dividend_yield_times", ctypes.c_void_p), ("n_dividend_yield_times", ctypes.c_uint64),
        ("cumulative_dividend_yields", ctypes.c_void_p), ("n_cumulative_dividend_yields", ctypes.c_uint64),
        ("dividend_nodes", ctypes.c_void_p), ("n_dividend_nodes", ctypes.c_uint64),
        ("dividend_amounts", ctypes.c_void_p), ("n_dividend_amounts", ctypes.c_uint64),
        ("exercise_nodes", ctypes.c_void_p), ("n_exercise_nodes", ctypes.c_uint64),
        ("expiry_node", ctypes.c_uint32),
        ("annualized_volatility", ctypes.c_double),
        ("dividend_policy", ctypes.c_int32),
        ("training_paths", ctypes.c_uint64),
        ("evaluation_paths", ctypes.c_uint64),
        ("training_seed", ctypes.c_uint64),
        ("training_domain", ctypes.c_uint32),
        ("evaluation_seed", ctypes.c_uint64),
        ("evaluation_domain", ctypes.c_uint32),
        ("polynomial_degree", ctypes.c_uint32),
        ("rank_tolerance", ctypes.c_double),
        ("condition_limit", ctypes.c_double),
        ("tie_rule", ctypes.c_int32),
        ("insufficient_exercise_support", ctypes.c_int32),
    ]


class FoLsmNodeDiagnostic(ctypes.Structure):
    _fields_ = [
        ("node", ctypes.c_uint32),
        ("kind", ctypes.c_int32),
        ("exercise", ctypes.c_int32),
        ("estimated_continuation", ctypes.c_double),
        ("in_the_money_paths", ctypes.c_uint32),
        ("observations", ctypes.c_uint64),
        ("columns", ctypes.c_uint64),
        ("rank", ctypes.c_uint64),
        ("condition_number", ctypes.c_double),
        ("predictor_mean", ctypes.c_double),
        ("predictor_scale", ctypes.c_double),
    ]


class FoLsmCallResult(ctypes.Structure):
    # Caller-owned buffers, given by address like the request's arrays.
    _fields_ = [
        ("price", ctypes.c_double),
        ("paths", ctypes.c_uint32),
        ("has_sample_standard_deviation", ctypes.c_int32),
        ("sample_standard_deviation", ctypes.c_double),
        ("has_standard_error", ctypes.c_int32),
        ("standard_error", ctypes.c_double),
        ("observation_nodes", ctypes.c_void_p), ("observation_capacity", ctypes.c_uint64),
        ("exercise_counts", ctypes.c_void_p),
        ("n_observations", ctypes.c_uint64),
        ("diagnostics", ctypes.c_void_p), ("diagnostics_capacity", ctypes.c_uint64),
        ("n_diagnostics", ctypes.c_uint64),
    ]


class FoLsmCallGreeks(ctypes.Structure):
    _fields_ = [
        ("delta", ctypes.c_double),
        ("vega", ctypes.c_double),
        ("log_discount_sensitivities", c_double_p), ("log_discount_capacity", ctypes.c_uint64),
        ("dividend_sensitivities", c_double_p), ("dividend_capacity", ctypes.c_uint64),
    ]


class FoLsmGroupedRequest(ctypes.Structure):
    _fields_ = [
        ("group_offsets", c_uint32_p), ("n_group_offsets", ctypes.c_uint64),
        ("initial_spots", c_double_p), ("n_initial_spots", ctypes.c_uint64),
        ("strikes", c_double_p), ("n_strikes", ctypes.c_uint64),
        ("maturities", c_double_p), ("n_maturities", ctypes.c_uint64),
        ("rates", c_double_p), ("n_rates", ctypes.c_uint64),
        ("volatilities", c_double_p), ("n_volatilities", ctypes.c_uint64),
        ("dividend_model", ctypes.c_int32),
        ("dividend_yields", c_double_p), ("n_dividend_yields", ctypes.c_uint64),
        ("dividend_offsets", c_int64_p), ("n_dividend_offsets", ctypes.c_uint64),
        ("dividend_times", c_double_p), ("n_dividend_times", ctypes.c_uint64),
        ("dividend_amounts", c_double_p), ("n_dividend_amounts", ctypes.c_uint64),
        ("dividend_policy", ctypes.c_int32),
        ("maturity_boundary", ctypes.c_int32),
        ("volatility_convention", ctypes.c_int32),
        ("exercise_mesh", ctypes.c_int32),
        ("has_base_intervals", ctypes.c_int32), ("base_intervals", ctypes.c_uint32),
        ("has_origin_exercise", ctypes.c_int32), ("origin_exercise", ctypes.c_int32),
        ("explicit_exercise_offsets", c_int64_p), ("n_explicit_exercise_offsets", ctypes.c_uint64),
        ("explicit_exercise_times", c_double_p), ("n_explicit_exercise_times", ctypes.c_uint64),
        ("training_paths", ctypes.c_uint64),
        ("evaluation_paths", ctypes.c_uint64),
        ("training_seed", ctypes.c_uint64),
        ("training_domain_start", ctypes.c_uint32),
        ("evaluation_seed", ctypes.c_uint64),
        ("evaluation_domain_start", ctypes.c_uint32),
        ("polynomial_degree", ctypes.c_uint32),
        ("rank_tolerance", ctypes.c_double),
        ("condition_limit", ctypes.c_double),
        ("tie_rule", ctypes.c_int32),
        ("insufficient_exercise_support", ctypes.c_int32),
    ]


class FoLsmRaggedRequest(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_uint64),
        ("initial_spots", c_double_p),
        ("strikes", c_double_p),
        ("maturities", c_double_p),
        ("rates", c_double_p),
        ("volatilities", c_double_p),
        ("dividend_yields", c_double_p),
        ("dividend_offsets", ctypes.POINTER(ctypes.c_int64)), ("n_dividend_offsets", ctypes.c_uint64),
        ("dividend_times", c_double_p), ("dividend_amounts", c_double_p), ("n_dividend_events", ctypes.c_uint64),
        ("dividend_policy", ctypes.c_int32),
        ("maturity_boundary", ctypes.c_int32),
        ("exercise_offsets", ctypes.POINTER(ctypes.c_int64)), ("n_exercise_offsets", ctypes.c_uint64),
        ("exercise_times", c_double_p), ("n_exercise_times", ctypes.c_uint64),
        ("origin_exercise", ctypes.c_int32),
        ("training_paths", ctypes.POINTER(ctypes.c_uint64)),
        ("evaluation_paths", ctypes.POINTER(ctypes.c_uint64)),
        ("training_seed", ctypes.c_uint64),
        ("training_domain_start", ctypes.c_uint32),
        ("evaluation_seed", ctypes.c_uint64),
        ("evaluation_domain_start", ctypes.c_uint32),
        ("polynomial_degree", ctypes.c_uint32),
        ("rank_tolerance", ctypes.c_double),
        ("condition_limit", ctypes.c_double),
        ("tie_rule", ctypes.c_int32),
        ("insufficient_exercise_support", ctypes.c_int32),
    ]


class FoRaggedGreeksColumns(ctypes.Structure):
    _fields_ = [
        ("delta", c_double_p),
        ("vega", c_double_p),
        ("log_discount_sensitivities", c_double_p), ("log_discount_capacity", ctypes.c_uint64),
        ("log_discount_offsets", ctypes.POINTER(ctypes.c_int64)),
        ("dividend_sensitivities", c_double_p),
    ]


class FoBatchResultColumns(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_uint64),
        ("prices", c_double_p),
        ("sample_standard_deviations", c_double_p),
        ("standard_errors", c_double_p),
        ("origin_decisions_fitted", c_uint8_p),
        ("origin_exercised", c_uint8_p),
        ("regression_nodes", c_uint32_p),
        ("no_training_support_nodes", c_uint32_p),
        ("insufficient_exercise_support_nodes", c_uint32_p),
        ("minimum_in_the_money_training_paths", c_uint32_p),
        ("maximum_regression_condition_numbers", c_double_p),
        ("early_exercise_paths", c_uint32_p),
        ("expiry_paths", c_uint32_p),
    ]


class FoGbmSeededRequest(ctypes.Structure):
    _fields_ = [
        ("initial_spot", ctypes.c_double),
        ("schedule_times", c_double_p), ("n_schedule_times", ctypes.c_uint64),
        ("curve_times", c_double_p), ("n_curve_times", ctypes.c_uint64),
        ("log_discounts", c_double_p), ("n_log_discounts", ctypes.c_uint64),
        ("dividend_yield_times", c_double_p), ("n_dividend_yield_times", ctypes.c_uint64),
        ("cumulative_dividend_yields", c_double_p), ("n_cumulative_dividend_yields", ctypes.c_uint64),
        ("dividend_nodes", c_uint32_p), ("n_dividend_nodes", ctypes.c_uint64),
        ("dividend_amounts", c_double_p), ("n_dividend_amounts", ctypes.c_uint64),
        ("exercise_nodes", c_uint32_p), ("n_exercise_nodes", ctypes.c_uint64),
        ("expiry_node", ctypes.c_uint32),
        ("annualized_volatility", ctypes.c_double),
        ("dividend_policy", ctypes.c_int32),
        ("paths", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("domain", ctypes.c_uint32),
    ]


class FoBatchTuning(ctypes.Structure):
    _fields_ = [("sim_blocks", ctypes.c_int32), ("eval_blocks", ctypes.c_int32), ("strikes", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("phases", ctypes.c_int32)]


class FoBatchLaunchInfo(ctypes.Structure):
    _fields_ = [("tuning", FoBatchTuning), ("source", ctypes.c_int32), ("grid", ctypes.c_int32),
                ("items", ctypes.c_uint64), ("tuning_launches", ctypes.c_uint64), ("graph_replays", ctypes.c_uint64),
                ("graph_captures", ctypes.c_uint64)]


PACKAGE_ROOT: Final = Path(__file__).resolve().parent
LIBRARY_PATH: Final = PACKAGE_ROOT / "_lib" / "libfinoptions_cuda.so"

# Every symbol include/finoptions_cuda.h declares (checked by the test suite against the header).
EXPORTED_SYMBOLS: Final = (
    "fo_cuda_executor_create",
    "fo_executor_destroy",
    "fo_executor_device",
    "fo_price_lsm_call_f64",
    "fo_lsm_call_plan_create",
    "fo_lsm_call_plan_launch",
    "fo_lsm_call_plan_collect",
    "fo_lsm_call_plan_time_launches",
    "fo_lsm_call_plan_transfer_bytes",
    "fo_lsm_call_plan_kernel_count",
    "fo_lsm_call_plan_stream",
    "fo_lsm_call_plan_destroy",
    "fo_price_lsm_call_f64_noalloc",
    "fo_price_lsm_call_greeks_f64",
    "fo_lsm_call_plan_set_greeks",
    "fo_lsm_call_plan_greeks",
    "fo_lsm_call_plan_revalue_f64",
    "fo_lsm_call_plan_stopping_rows",
    "fo_price_lsm_grouped_f64",
    "fo_price_lsm_batch_f64",
    "fo_price_lsm_ragged_f64",
    "fo_executor_batch_kernel_ms",
    "fo_executor_batch_transfer_bytes",
    "fo_executor_set_batch_tuning",
    "fo_executor_batch_launch",
    "fo_simulate_gbm_seeded_f64",
    "fo_simulate_gbm_f64",
    "fo_simulate_gbm_device_f64",
    "fo_sample_standard_normals_f64",
    "fo_build_info",
    "fo_validate_lsm_grouped_f64",
    "fo_validate_lsm_ragged_f64",
)

_library: ctypes.CDLL | None = None


def _declare(lib: ctypes.CDLL) -> None:
    vp = ctypes.c_void_p
    err = ctypes.POINTER(FoError)
    lib.fo_cuda_executor_create.argtypes = [ctypes.c_int32, ctypes.POINTER(vp), err]
    lib.fo_cuda_executor_create.restype = ctypes.c_int
    lib.fo_executor_destroy.argtypes = [vp]
    lib.fo_executor_destroy.restype = None
    lib.fo_executor_device.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    lib.fo_executor_device.restype = ctypes.c_int
    lib.fo_price_lsm_call_f64.argtypes = [vp, ctypes.POINTER(FoLsmCallRequest), ctypes.POINTER(FoLsmCallResult), err]
    lib.fo_price_lsm_call_f64.restype = ctypes.c_int
    lib.fo_price_lsm_call_f64_noalloc.argtypes = [ctypes.POINTER(FoLsmCallRequest), vp, ctypes.POINTER(FoLsmCallResult), err]
    lib.fo_price_lsm_call_f64_noalloc.restype = ctypes.c_int
    lib.fo_lsm_call_plan_create.argtypes = [vp, ctypes.POINTER(FoLsmCallRequest), ctypes.POINTER(vp), err]
    lib.fo_lsm_call_plan_create.restype = ctypes.c_int
    lib.fo_lsm_call_plan_launch.argtypes = [vp, err]
    lib.fo_lsm_call_plan_launch.restype = ctypes.c_int
    lib.fo_lsm_call_plan_collect.argtypes = [vp, ctypes.POINTER(FoLsmCallResult), err]
    lib.fo_lsm_call_plan_collect.restype = ctypes.c_int
    lib.fo_lsm_call_plan_time_launches.argtypes = [vp, ctypes.c_uint32, c_double_p, c_double_p, ctypes.c_uint64, err]
    lib.fo_lsm_call_plan_time_launches.restype = ctypes.c_int
    lib.fo_lsm_call_plan_transfer_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    lib.fo_lsm_call_plan_transfer_bytes.restype = ctypes.c_int
    lib.fo_lsm_call_plan_kernel_count.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    lib.fo_lsm_call_plan_kernel_count.restype = ctypes.c_int
    lib.fo_lsm_call_plan_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.fo_lsm_call_plan_stream.restype = ctypes.c_int
    greeks = ctypes.POINTER(FoLsmCallGreeks)
    lib.fo_price_lsm_call_greeks_f64.argtypes = [vp, ctypes.POINTER(FoLsmCallRequest), ctypes.POINTER(FoLsmCallResult),
                                                 greeks, err]
    lib.fo_price_lsm_call_greeks_f64.restype = ctypes.c_int
    lib.fo_lsm_call_plan_set_greeks.argtypes = [vp, ctypes.c_int32, err]
    lib.fo_lsm_call_plan_set_greeks.restype = ctypes.c_int
    lib.fo_lsm_call_plan_greeks.argtypes = [vp, greeks, err]
    lib.fo_lsm_call_plan_greeks.restype = ctypes.c_int
    lib.fo_lsm_call_plan_revalue_f64.argtypes = [vp, ctypes.POINTER(FoLsmCallRequest), ctypes.POINTER(FoLsmCallResult), err]
    lib.fo_lsm_call_plan_revalue_f64.restype = ctypes.c_int
    lib.fo_lsm_call_plan_stopping_rows.argtypes = [vp, ctypes.c_void_p, ctypes.c_uint64, err]
    lib.fo_lsm_call_plan_stopping_rows.restype = ctypes.c_int
    lib.fo_lsm_call_plan_destroy.argtypes = [vp]
    lib.fo_lsm_call_plan_destroy.restype = None
    for name in ("fo_price_lsm_grouped_f64", "fo_price_lsm_batch_f64"):
        fn = getattr(lib, name)
        fn.argtypes = [vp, ctypes.POINTER(FoLsmGroupedRequest), ctypes.POINTER(FoBatchResultColumns), err]
        fn.restype = ctypes.c_int
    lib.fo_price_lsm_ragged_f64.argtypes = [vp, ctypes.POINTER(FoLsmRaggedRequest), ctypes.POINTER(FoBatchResultColumns),
                                            ctypes.POINTER(FoRaggedGreeksColumns), err]
    lib.fo_price_lsm_ragged_f64.restype = ctypes.c_int
    lib.fo_executor_batch_kernel_ms.argtypes = [vp, c_double_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    lib.fo_executor_batch_kernel_ms.restype = ctypes.c_int
    u64p = ctypes.POINTER(ctypes.c_uint64)
    lib.fo_executor_batch_transfer_bytes.argtypes = [vp, u64p, u64p]
    lib.fo_executor_batch_transfer_bytes.restype = ctypes.c_int
    lib.fo_executor_set_batch_tuning.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(FoBatchTuning), err]
    lib.fo_executor_set_batch_tuning.restype = ctypes.c_int
    lib.fo_executor_batch_launch.argtypes = [vp, ctypes.POINTER(FoBatchLaunchInfo)]
    lib.fo_executor_batch_launch.restype = ctypes.c_int
    lib.fo_simulate_gbm_seeded_f64.argtypes = [vp, ctypes.POINTER(FoGbmSeededRequest), c_double_p, ctypes.c_uint64, err]
    lib.fo_simulate_gbm_seeded_f64.restype = ctypes.c_int
    lib.fo_simulate_gbm_f64.argtypes = [vp, ctypes.POINTER(FoGbmSeededRequest), c_double_p, ctypes.c_uint64,
                                        c_double_p, ctypes.c_uint64, err]
    lib.fo_simulate_gbm_f64.restype = ctypes.c_int
    lib.fo_simulate_gbm_device_f64.argtypes = [vp, ctypes.POINTER(FoGbmSeededRequest), vp, ctypes.c_uint64, vp,
                                               ctypes.c_uint64, err]
    lib.fo_simulate_gbm_device_f64.restype = ctypes.c_int
    lib.fo_sample_standard_normals_f64.argtypes = [
        vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
        c_double_p, ctypes.c_uint64, err,
    ]
    lib.fo_sample_standard_normals_f64.restype = ctypes.c_int
    lib.fo_validate_lsm_grouped_f64.argtypes = [ctypes.POINTER(FoLsmGroupedRequest), ctypes.c_int32, err]
    lib.fo_validate_lsm_grouped_f64.restype = ctypes.c_int
    lib.fo_validate_lsm_ragged_f64.argtypes = [ctypes.POINTER(FoLsmRaggedRequest), err]
    lib.fo_validate_lsm_ragged_f64.restype = ctypes.c_int
    lib.fo_build_info.argtypes = [ctypes.c_char_p, ctypes.c_uint64]
    lib.fo_build_info.restype = ctypes.c_int


def library_path() -> Path:
    """Return the in-tree shared library path (overridable with FINOPTIONS_CUDA_LIBRARY)."""
    override = os.environ.get("FINOPTIONS_CUDA_LIBRARY")
    return Path(override) if override else LIBRARY_PATH


def load() -> ctypes.CDLL:
    """Load (once) and return the engine's shared library, failing loudly when it is missing."""
    global _library  # noqa: PLW0603 - process-wide handle to one shared library
    if _library is None:
        path = library_path()
        if not path.is_file():
            from ._errors import ExecutionError  # noqa: PLC0415 - avoid an import cycle

            msg = (
                f"the B200 engine library {path} is not built; run "
                "`python finoptions-engine_b200/build.py` (there is no CPU fallback)"
            )
            raise ExecutionError(msg)
        lib = ctypes.CDLL(str(path))
        _declare(lib)
        _library = lib
    return _library
