"""Native surface of the B200 engine: the reference's ``finoptions._native`` LSM functions.

Every function here keeps the name, argument order and meaning of the reference's PyO3 function
(crates/finoptions-python/src/lib.rs) and calls the engine's C ABI (include/finoptions_cuda.h)
through ctypes. String enums are parsed exactly as the reference parses them (lib.rs:514-556).
The executor argument is a ``CudaExecutor`` handle; there is no CPU engine behind this module.
"""

from __future__ import annotations

import ctypes
import threading
from typing import Any, Final

import numpy as np

from . import _abi
from ._errors import BatchError, ExecutionError, InputError, LsmError, SimulationError, raise_for
from ._requests import (
    batch_columns,
    gbm_seeded_request,
    lsm_call_greeks,
    lsm_call_request,
    lsm_call_result,
    lsm_grouped_request,
    lsm_ragged_request,
)

__all__ = [
    "BatchError",
    "CudaExecutor",
    "ExecutionError",
    "InputError",
    "LsmError",
    "SimulationError",
    "build_info",
    "price_lsm_call_batch_cash_dividends_f64",
    "price_lsm_call_batch_continuous_yield_f64",
    "price_lsm_call_batch_escrowed_cash_dividends_f64",
    "price_lsm_call_grouped_batch_cash_dividends_f64",
    "price_lsm_call_grouped_batch_continuous_yield_f64",
    "price_lsm_call_grouped_batch_escrowed_cash_dividends_f64",
    "price_lsm_call_seeded_f64",
    "simulate_gbm_seeded_f64",
    "validate_cash_dividend_amount",
    "validate_constant_volatility",
    "validate_cumulative_dividend_yield_curve",
    "validate_event_schedule",
    "validate_log_discount_curve",
    "validate_ragged_cash_dividends_f64",
    "validate_ragged_exercise_times_f64",
]

_DIVIDEND_POLICIES: Final = {"liquidator": 0, "survivor": 1}
_TIE_RULES: Final = {"strictly_greater": 0, "greater_or_equal": 1}
_SUPPORT: Final = {"fail": 0, "continue": 1}
_ORIGIN: Final = {"excluded": 0, "included": 1}
_MATURITY: Final = {"strictly_before": 0, "at_or_before": 1}
_ESCROWED_VOL: Final = {"prepaid_forward": 0, "spot_matched_at_origin": 1}
_MESHES: Final = {"uniform": 0, "cash_dividend_dates": 1, "explicit_times": 2}
_FO_CODE_UNSUPPORTED_ENUM: Final = 125


def _lib() -> ctypes.CDLL:
    return _abi.load()


def _check(status: int, error: _abi.FoError) -> None:
    raise_for(status, error)


def _parse(table: dict[str, int], value: str, what: str, exc: type[Exception] = InputError) -> int:
    if value not in table:
        msg = f'unsupported {what} "{value}"'
        raise exc(msg)
    return table[value]


def _lib_validate(fn_name: str, *args: Any) -> None:
    lib = _lib()
    fn = getattr(lib, fn_name)
    err = _abi.FoError()
    status = fn(*args, ctypes.byref(err))
    _check(status, err)


def _f64_array(values: Any) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.float64))


def _u32_array(values: Any) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.uint32))


def _dp(array: np.ndarray) -> Any:
    return array.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _up(array: np.ndarray) -> Any:
    return array.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _ip(array: np.ndarray) -> Any:
    return array.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


class CudaExecutor:
    """One sm_100 device with its stream and device arena (the engine's fo_executor).

    Construction fails with ExecutionError when no Blackwell B200 device is available; nothing
    falls back to a CPU implementation.
    """

    def __init__(self, device: int = 0) -> None:
        lib = _lib()
        handle = ctypes.c_void_p()
        err = _abi.FoError()
        status = lib.fo_cuda_executor_create(int(device), ctypes.byref(handle), ctypes.byref(err))
        _check(status, err)
        self._handle = handle
        self._device = int(device)
        self._lock = threading.Lock()

    @property
    def device(self) -> int:
        return self._device

    @property
    def raw(self) -> ctypes.c_void_p:
        return self._handle

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            try:
                _lib().fo_executor_destroy(handle)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self._handle = ctypes.c_void_p()


def build_info() -> tuple[str, str]:
    """(package_version, compiler identity) like lib.rs:400-404."""
    buf = ctypes.create_string_buffer(256)
    _lib().fo_build_info(buf, len(buf))
    version, _, compiler = buf.value.decode().partition(";")
    return version, compiler


# ---- validation (lib.rs:405-473) ------------------------------------------------------------------


def validate_cash_dividend_amount(amount: float) -> None:
    _lib().fo_validate_cash_dividend_amount.argtypes = [ctypes.c_double, ctypes.POINTER(_abi.FoError)]
    _lib_validate("fo_validate_cash_dividend_amount", ctypes.c_double(amount))


def validate_constant_volatility(annualized_decimal: float) -> None:
    _lib().fo_validate_constant_volatility.argtypes = [ctypes.c_double, ctypes.POINTER(_abi.FoError)]
    _lib_validate("fo_validate_constant_volatility", ctypes.c_double(annualized_decimal))


def validate_event_schedule(
    times: list[float],
    dividend_nodes: list[int],
    dividend_amounts: list[float],
    exercise_nodes: list[int],
    expiry_node: int,
) -> None:
    t, dn, da, en = _f64_array(times), _u32_array(dividend_nodes), _f64_array(dividend_amounts), _u32_array(exercise_nodes)
    _lib_validate("fo_validate_event_schedule", _dp(t), ctypes.c_uint64(t.size), _up(dn), ctypes.c_uint64(dn.size),
                  _dp(da), ctypes.c_uint64(da.size), _up(en), ctypes.c_uint64(en.size), ctypes.c_uint32(expiry_node))


def validate_log_discount_curve(times: list[float], log_discounts: list[float]) -> None:
    t, v = _f64_array(times), _f64_array(log_discounts)
    _lib_validate("fo_validate_log_discount_curve", _dp(t), ctypes.c_uint64(t.size), _dp(v), ctypes.c_uint64(v.size))


def validate_cumulative_dividend_yield_curve(times: list[float], cumulative_yields: list[float]) -> None:
    t, v = _f64_array(times), _f64_array(cumulative_yields)
    _lib_validate("fo_validate_cumulative_dividend_yield_curve", _dp(t), ctypes.c_uint64(t.size), _dp(v),
                  ctypes.c_uint64(v.size))


def validate_ragged_cash_dividends_f64(offsets: np.ndarray, times: np.ndarray, amounts: np.ndarray) -> None:
    _lib_validate("fo_validate_ragged_cash_dividends", _ip(offsets), ctypes.c_uint64(offsets.size), _dp(times),
                  ctypes.c_uint64(times.size), _dp(amounts), ctypes.c_uint64(amounts.size))


def validate_ragged_exercise_times_f64(offsets: np.ndarray, times: np.ndarray) -> None:
    _lib_validate("fo_validate_ragged_exercise_times", _ip(offsets), ctypes.c_uint64(offsets.size), _dp(times),
                  ctypes.c_uint64(times.size))


# ---- pricing ----------------------------------------------------------------------------------


def _executor_handle(executor: object) -> ctypes.c_void_p:
    if not isinstance(executor, CudaExecutor):
        msg = "the B200 engine prices only on a CudaExecutor"
        raise ExecutionError(msg)
    return executor.raw


def price_lsm_call_seeded_result_f64(  # noqa: PLR0913 - price_lsm_call_seeded_f64's signature
    initial_spot: float,
    strike: float,
    schedule_times: list[float],
    curve_times: list[float],
    log_discounts: list[float],
    dividend_yield_times: list[float],
    cumulative_dividend_yields: list[float],
    dividend_nodes: list[int],
    dividend_amounts: list[float],
    exercise_nodes: list[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: str,
    executor: CudaExecutor,
    training_paths: int,
    evaluation_paths: int,
    training_seed: int,
    training_domain: int,
    evaluation_seed: int,
    evaluation_domain: int,
    polynomial_degree: int,
    rank_tolerance: float,
    condition_limit: float,
    tie_rule: str,
    insufficient_exercise_support: str,
) -> tuple:
    """price_lsm_call_seeded_f64 returning the caller-owned result buffers (a CallResult) instead of
    the NativeLsmResult tuple; the public pricing call builds its records straight from them."""
    handle = _executor_handle(executor)
    request = lsm_call_request(
        initial_spot=initial_spot,
        strike=strike,
        schedule_times=schedule_times,
        curve_times=curve_times,
        log_discounts=log_discounts,
        dividend_yield_times=dividend_yield_times,
        cumulative_dividend_yields=cumulative_dividend_yields,
        dividend_nodes=dividend_nodes,
        dividend_amounts=dividend_amounts,
        exercise_nodes=exercise_nodes,
        expiry_node=expiry_node,
        annualized_volatility=annualized_volatility,
        dividend_policy=_DIVIDEND_POLICIES.get(dividend_policy, -1),
        training_paths=training_paths,
        evaluation_paths=evaluation_paths,
        training_seed=training_seed,
        training_domain=training_domain,
        evaluation_seed=evaluation_seed,
        evaluation_domain=evaluation_domain,
        polynomial_degree=polynomial_degree,
        rank_tolerance=rank_tolerance,
        condition_limit=condition_limit,
        tie_rule=_TIE_RULES.get(tie_rule, -1),
        insufficient_exercise_support=_SUPPORT.get(insufficient_exercise_support, -1),
    )
    result = lsm_call_result(request.exercise_rows)
    err = _abi.FoError()
    status = _lib().fo_price_lsm_call_f64(handle, ctypes.byref(request.struct), ctypes.byref(result.struct),
                                          ctypes.byref(err))
    if status and err.code == _FO_CODE_UNSUPPORTED_ENUM:
        # The C ABI carries integer enums; report the caller's string like lib.rs:514-556.
        message = err.message.decode()
        for prefix, value in (("unsupported dividend policy", dividend_policy),
                              ("unsupported exercise tie rule", tie_rule),
                              ("unsupported insufficient exercise support policy", insufficient_exercise_support)):
            if message.startswith(prefix):
                raise InputError(f'{prefix} "{value}"')
    _check(status, err)
    return result


def price_lsm_call_seeded_f64(  # noqa: PLR0913 - mirrors the reference's native signature
    initial_spot: float,
    strike: float,
    schedule_times: list[float],
    curve_times: list[float],
    log_discounts: list[float],
    dividend_yield_times: list[float],
    cumulative_dividend_yields: list[float],
    dividend_nodes: list[int],
    dividend_amounts: list[float],
    exercise_nodes: list[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: str,
    executor: CudaExecutor,
    training_paths: int,
    evaluation_paths: int,
    training_seed: int,
    training_domain: int,
    evaluation_seed: int,
    evaluation_domain: int,
    polynomial_degree: int,
    rank_tolerance: float,
    condition_limit: float,
    tie_rule: str,
    insufficient_exercise_support: str,
) -> tuple:
    """NativeLsmResult of one seeded single-contract LSM price (lib.rs:1169-1241)."""
    return price_lsm_call_seeded_result_f64(
        initial_spot, strike, schedule_times, curve_times, log_discounts, dividend_yield_times,
        cumulative_dividend_yields, dividend_nodes, dividend_amounts, exercise_nodes, expiry_node,
        annualized_volatility, dividend_policy, executor, training_paths, evaluation_paths, training_seed,
        training_domain, evaluation_seed, evaluation_domain, polynomial_degree, rank_tolerance, condition_limit,
        tie_rule, insufficient_exercise_support,
    ).as_tuple()


def price_lsm_call_greeks_seeded_f64(  # noqa: PLR0913 - price_lsm_call_seeded_f64's signature
    initial_spot: float,
    strike: float,
    schedule_times: list[float],
    curve_times: list[float],
    log_discounts: list[float],
    dividend_yield_times: list[float],
    cumulative_dividend_yields: list[float],
    dividend_nodes: list[int],
    dividend_amounts: list[float],
    exercise_nodes: list[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: str,
    executor: CudaExecutor,
    training_paths: int,
    evaluation_paths: int,
    training_seed: int,
    training_domain: int,
    evaluation_seed: int,
    evaluation_domain: int,
    polynomial_degree: int,
    rank_tolerance: float,
    condition_limit: float,
    tie_rule: str,
    insufficient_exercise_support: str,
) -> tuple:
    """(NativeLsmResult, delta, vega, dP/dL per node, dP/dD per cash dividend) of the same request
    as price_lsm_call_seeded_f64: the fixed-policy pathwise adjoint, formed in the pricing pass."""
    handle = _executor_handle(executor)
    request = lsm_call_request(
        initial_spot=initial_spot, strike=strike, schedule_times=schedule_times, curve_times=curve_times,
        log_discounts=log_discounts, dividend_yield_times=dividend_yield_times,
        cumulative_dividend_yields=cumulative_dividend_yields, dividend_nodes=dividend_nodes,
        dividend_amounts=dividend_amounts, exercise_nodes=exercise_nodes, expiry_node=expiry_node,
        annualized_volatility=annualized_volatility, dividend_policy=_DIVIDEND_POLICIES.get(dividend_policy, -1),
        training_paths=training_paths, evaluation_paths=evaluation_paths, training_seed=training_seed,
        training_domain=training_domain, evaluation_seed=evaluation_seed, evaluation_domain=evaluation_domain,
        polynomial_degree=polynomial_degree, rank_tolerance=rank_tolerance, condition_limit=condition_limit,
        tie_rule=_TIE_RULES.get(tie_rule, -1),
        insufficient_exercise_support=_SUPPORT.get(insufficient_exercise_support, -1),
    )
    result = lsm_call_result(request.exercise_rows)
    greeks, d_log_discounts, d_dividends = lsm_call_greeks(len(schedule_times), len(dividend_nodes))
    err = _abi.FoError()
    status = _lib().fo_price_lsm_call_greeks_f64(handle, ctypes.byref(request.struct), ctypes.byref(result.struct),
                                                 ctypes.byref(greeks), ctypes.byref(err))
    _check(status, err)
    return (result.as_tuple(), greeks.delta, greeks.vega, d_log_discounts.tolist(), d_dividends.tolist())


def simulate_gbm_seeded_f64(  # noqa: PLR0913 - mirrors the reference's native signature
    initial_spot: float,
    schedule_times: list[float],
    curve_times: list[float],
    log_discounts: list[float],
    dividend_yield_times: list[float],
    cumulative_dividend_yields: list[float],
    dividend_nodes: list[int],
    dividend_amounts: list[float],
    exercise_nodes: list[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: str,
    executor: CudaExecutor,
    paths: int,
    seed: int,
    domain: int,
) -> np.ndarray:
    """Time-major [observations, paths] seeded GBM states (lib.rs:1019-1058)."""
    handle = _executor_handle(executor)
    policy = _parse(_DIVIDEND_POLICIES, dividend_policy, "dividend policy")
    request = gbm_seeded_request(
        initial_spot=initial_spot,
        schedule_times=schedule_times,
        curve_times=curve_times,
        log_discounts=log_discounts,
        dividend_yield_times=dividend_yield_times,
        cumulative_dividend_yields=cumulative_dividend_yields,
        dividend_nodes=dividend_nodes,
        dividend_amounts=dividend_amounts,
        exercise_nodes=exercise_nodes,
        expiry_node=expiry_node,
        annualized_volatility=annualized_volatility,
        dividend_policy=policy,
        paths=paths,
        seed=seed,
        domain=domain,
    )
    out = np.empty((request.rows, paths), dtype=np.float64)
    err = _abi.FoError()
    status = _lib().fo_simulate_gbm_seeded_f64(handle, ctypes.byref(request.struct), _dp(out), ctypes.c_uint64(out.size),
                                               ctypes.byref(err))
    _check(status, err)
    return out



def _gbm_request(initial_spot, schedule_times, curve_times, log_discounts, dividend_yield_times,
                 cumulative_dividend_yields, dividend_nodes, dividend_amounts, exercise_nodes, expiry_node,
                 annualized_volatility, dividend_policy, paths, seed=0, domain=0):
    return gbm_seeded_request(
        initial_spot=initial_spot, schedule_times=schedule_times, curve_times=curve_times,
        log_discounts=log_discounts, dividend_yield_times=dividend_yield_times,
        cumulative_dividend_yields=cumulative_dividend_yields, dividend_nodes=dividend_nodes,
        dividend_amounts=dividend_amounts, exercise_nodes=exercise_nodes, expiry_node=expiry_node,
        annualized_volatility=annualized_volatility,
        dividend_policy=_parse(_DIVIDEND_POLICIES, dividend_policy, "dividend policy"), paths=paths, seed=seed,
        domain=domain)


def simulate_gbm_f64(  # noqa: PLR0913 - mirrors the reference's native signature
    initial_spot: float,
    schedule_times: list[float],
    curve_times: list[float],
    log_discounts: list[float],
    dividend_yield_times: list[float],
    cumulative_dividend_yields: list[float],
    dividend_nodes: list[int],
    dividend_amounts: list[float],
    exercise_nodes: list[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: str,
    executor: CudaExecutor,
    normals: np.ndarray,
) -> np.ndarray:
    """Time-major [observations, paths] GBM states driven by caller normals [intervals, paths]
    (simulate_gbm_f64, lib.rs:969-1018)."""
    handle = _executor_handle(executor)
    rows, paths = (int(n) for n in normals.shape)
    request = _gbm_request(initial_spot, schedule_times, curve_times, log_discounts, dividend_yield_times,
                           cumulative_dividend_yields, dividend_nodes, dividend_amounts, exercise_nodes, expiry_node,
                           annualized_volatility, dividend_policy, paths)
    out = np.empty((request.rows, paths), dtype=np.float64)
    err = _abi.FoError()
    # A one-element stand-in keeps the pointer valid for an empty matrix (the engine rejects it first).
    source = normals if normals.size else np.zeros(1)
    status = _lib().fo_simulate_gbm_f64(handle, ctypes.byref(request.struct), _dp(source), ctypes.c_uint64(rows),
                                        _dp(out) if out.size else None, ctypes.c_uint64(out.size), ctypes.byref(err))
    _check(status, err)
    return out


def simulate_gbm_device_f64(  # noqa: PLR0913 - the simulation arguments plus the device buffers
    initial_spot: float,
    schedule_times: list[float],
    curve_times: list[float],
    log_discounts: list[float],
    dividend_yield_times: list[float],
    cumulative_dividend_yields: list[float],
    dividend_nodes: list[int],
    dividend_amounts: list[float],
    exercise_nodes: list[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: str,
    executor: CudaExecutor,
    paths: int,
    seed: int = 0,
    domain: int = 0,
    normals: Any = None,
) -> Any:
    """The states as a torch.float64 tensor [observations, paths] on the executor's device, written
    there by the kernel (no host copy): from the Philox streams (seed, domain), or from `normals`,
    a C-contiguous torch.float64 tensor [intervals, paths] on the same device."""
    import torch  # noqa: PLC0415 - only device-tensor callers need torch

    handle = _executor_handle(executor)
    device = torch.device("cuda", executor.device)
    if normals is not None:
        if (not isinstance(normals, torch.Tensor) or normals.dtype != torch.float64 or normals.device != device
                or normals.dim() != 2 or not normals.is_contiguous()):
            raise InputError(f"normals must be a C-contiguous torch.float64 [intervals, paths] tensor on {device}")
        paths = int(normals.shape[1])
    request = _gbm_request(initial_spot, schedule_times, curve_times, log_discounts, dividend_yield_times,
                           cumulative_dividend_yields, dividend_nodes, dividend_amounts, exercise_nodes, expiry_node,
                           annualized_volatility, dividend_policy, paths, seed, domain)
    out = torch.empty((request.rows, paths), dtype=torch.float64, device=device)
    # Work queued on torch's stream (the normals, the output's allocation) finishes before the
    # executor's stream reads or writes them; the call returns once the states are written.
    torch.cuda.current_stream(device).synchronize()
    err = _abi.FoError()
    status = _lib().fo_simulate_gbm_device_f64(
        handle, ctypes.byref(request.struct), None if normals is None else ctypes.c_void_p(normals.data_ptr()),
        ctypes.c_uint64(0 if normals is None else normals.shape[0]), ctypes.c_void_p(out.data_ptr()),
        ctypes.c_uint64(out.numel()), ctypes.byref(err))
    _check(status, err)
    return out


def _method(
    exercise_mesh: str,
    base_intervals: int | None,
    origin_exercise: str | None,
    explicit_exercise_offsets: np.ndarray | None,
    explicit_exercise_times: np.ndarray | None,
) -> dict[str, Any]:
    # parse_batch_lsm_method (lib.rs:1302-1415): field presence rules per mesh
    mesh = _parse(_MESHES, exercise_mesh, "batched LSM exercise mesh")
    if mesh == 0:
        if explicit_exercise_offsets is not None or explicit_exercise_times is not None:
            raise InputError("uniform exercise mesh forbids explicit exercise buffers")
        if base_intervals is None:
            raise InputError("uniform exercise mesh requires base_intervals")
        if origin_exercise is None:
            raise InputError("uniform exercise mesh requires origin_exercise")
    elif mesh == 1:
        if (base_intervals is not None or origin_exercise is not None or explicit_exercise_offsets is not None
                or explicit_exercise_times is not None):
            raise InputError("cash-dividend-date exercise mesh forbids uniform and explicit mesh fields")
    else:
        if base_intervals is not None:
            raise InputError("explicit exercise mesh forbids base_intervals")
        if origin_exercise is None:
            raise InputError("explicit exercise mesh requires origin_exercise")
        if explicit_exercise_offsets is None:
            raise InputError("explicit exercise mesh requires exercise offsets")
        if explicit_exercise_times is None:
            raise InputError("explicit exercise mesh requires exercise times")
    return {
        "exercise_mesh": mesh,
        "base_intervals": base_intervals,
        "origin_exercise": None if origin_exercise is None else _parse(_ORIGIN, origin_exercise,
                                                                      "origin exercise convention"),
        "explicit_exercise_offsets": explicit_exercise_offsets,
        "explicit_exercise_times": explicit_exercise_times,
    }


def _grouped(  # noqa: PLR0913
    entry: str,
    group_offsets: np.ndarray | None,
    initial_spots: np.ndarray,
    strikes: np.ndarray,
    maturities: np.ndarray,
    rates: np.ndarray,
    volatilities: np.ndarray,
    dividends: dict[str, Any],
    mesh: dict[str, Any],
    executor: CudaExecutor,
    training_paths: int,
    evaluation_paths: int,
    training_seed: int,
    training_domain_start: int,
    evaluation_seed: int,
    evaluation_domain_start: int,
    polynomial_degree: int,
    rank_tolerance: float,
    condition_limit: float,
    tie_rule: str,
    insufficient_exercise_support: str,
) -> tuple | None:
    # executor None: run the whole-request validation only (no device is touched).
    handle = None if executor is None else _executor_handle(executor)
    tie = _parse(_TIE_RULES, tie_rule, "exercise tie rule")
    support = _parse(_SUPPORT, insufficient_exercise_support, "insufficient exercise support policy")
    request = lsm_grouped_request(
        group_offsets=group_offsets,
        initial_spots=initial_spots,
        strikes=strikes,
        maturities=maturities,
        rates=rates,
        volatilities=volatilities,
        training_paths=training_paths,
        evaluation_paths=evaluation_paths,
        training_seed=training_seed,
        training_domain_start=training_domain_start,
        evaluation_seed=evaluation_seed,
        evaluation_domain_start=evaluation_domain_start,
        polynomial_degree=polynomial_degree,
        rank_tolerance=rank_tolerance,
        condition_limit=condition_limit,
        tie_rule=tie,
        insufficient_exercise_support=support,
        **dividends,
        **mesh,
    )
    err = _abi.FoError()
    if handle is None:
        grouped = 1 if entry == "fo_price_lsm_grouped_f64" else 0
        _check(_lib().fo_validate_lsm_grouped_f64(ctypes.byref(request.struct), grouped, ctypes.byref(err)), err)
        return None
    columns = batch_columns(request.rows)
    status = getattr(_lib(), entry)(handle, ctypes.byref(request.struct), ctypes.byref(columns.struct),
                                    ctypes.byref(err))
    _check(status, err)
    return columns.as_tuple()


def _cash(offsets: np.ndarray, times: np.ndarray, amounts: np.ndarray, model: int, **extra: int) -> dict[str, Any]:
    return {"dividend_model": model, "dividend_offsets": offsets, "dividend_times": times,
            "dividend_amounts": amounts, **extra}


def price_lsm_call_grouped_batch_continuous_yield_f64(  # noqa: PLR0913
    group_offsets, initial_spots, strikes, maturities, rates, volatilities, annualized_dividend_yields,
    exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times,
    executor, training_paths, evaluation_paths, training_seed, training_domain_start, evaluation_seed,
    evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit, tie_rule,
    insufficient_exercise_support,
) -> tuple:
    mesh = _method(exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times)
    return _grouped("fo_price_lsm_grouped_f64", group_offsets, initial_spots, strikes, maturities, rates,
                    volatilities, {"dividend_model": 0, "dividend_yields": annualized_dividend_yields}, mesh, executor,
                    training_paths, evaluation_paths, training_seed, training_domain_start, evaluation_seed,
                    evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit, tie_rule,
                    insufficient_exercise_support)


def price_lsm_call_grouped_batch_cash_dividends_f64(  # noqa: PLR0913
    group_offsets, initial_spots, strikes, maturities, rates, volatilities, dividend_offsets, dividend_times,
    dividend_amounts, dividend_policy, maturity_boundary, exercise_mesh, base_intervals, origin_exercise,
    explicit_exercise_offsets, explicit_exercise_times, executor, training_paths, evaluation_paths, training_seed,
    training_domain_start, evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance,
    condition_limit, tie_rule, insufficient_exercise_support,
) -> tuple:
    policy = _parse(_DIVIDEND_POLICIES, dividend_policy, "dividend policy")
    boundary = _parse(_MATURITY, maturity_boundary, "maturity boundary", BatchError)
    mesh = _method(exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times)
    return _grouped("fo_price_lsm_grouped_f64", group_offsets, initial_spots, strikes, maturities, rates,
                    volatilities, _cash(dividend_offsets, dividend_times, dividend_amounts, 1,
                                        dividend_policy=policy, maturity_boundary=boundary),
                    mesh, executor, training_paths, evaluation_paths, training_seed, training_domain_start,
                    evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit,
                    tie_rule, insufficient_exercise_support)


def price_lsm_call_grouped_batch_escrowed_cash_dividends_f64(  # noqa: PLR0913
    group_offsets, initial_spots, strikes, maturities, rates, volatilities, dividend_offsets, dividend_times,
    dividend_amounts, volatility_convention, maturity_boundary, exercise_mesh, base_intervals, origin_exercise,
    explicit_exercise_offsets, explicit_exercise_times, executor, training_paths, evaluation_paths, training_seed,
    training_domain_start, evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance,
    condition_limit, tie_rule, insufficient_exercise_support,
) -> tuple:
    convention = _parse(_ESCROWED_VOL, volatility_convention, "escrowed volatility convention")
    boundary = _parse(_MATURITY, maturity_boundary, "maturity boundary", BatchError)
    mesh = _method(exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times)
    return _grouped("fo_price_lsm_grouped_f64", group_offsets, initial_spots, strikes, maturities, rates,
                    volatilities, _cash(dividend_offsets, dividend_times, dividend_amounts, 2,
                                        volatility_convention=convention, maturity_boundary=boundary),
                    mesh, executor, training_paths, evaluation_paths, training_seed, training_domain_start,
                    evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit,
                    tie_rule, insufficient_exercise_support)


def price_lsm_call_batch_continuous_yield_f64(  # noqa: PLR0913
    initial_spots, strikes, maturities, rates, volatilities, annualized_dividend_yields, exercise_mesh,
    base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times, executor, training_paths,
    evaluation_paths, training_seed, training_domain_start, evaluation_seed, evaluation_domain_start,
    polynomial_degree, rank_tolerance, condition_limit, tie_rule, insufficient_exercise_support,
) -> tuple:
    mesh = _method(exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times)
    return _grouped("fo_price_lsm_batch_f64", None, initial_spots, strikes, maturities, rates, volatilities,
                    {"dividend_model": 0, "dividend_yields": annualized_dividend_yields}, mesh, executor,
                    training_paths, evaluation_paths, training_seed, training_domain_start, evaluation_seed,
                    evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit, tie_rule,
                    insufficient_exercise_support)


def price_lsm_call_batch_cash_dividends_f64(  # noqa: PLR0913
    initial_spots, strikes, maturities, rates, volatilities, dividend_offsets, dividend_times, dividend_amounts,
    dividend_policy, maturity_boundary, exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets,
    explicit_exercise_times, executor, training_paths, evaluation_paths, training_seed, training_domain_start,
    evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit, tie_rule,
    insufficient_exercise_support,
) -> tuple:
    policy = _parse(_DIVIDEND_POLICIES, dividend_policy, "dividend policy")
    boundary = _parse(_MATURITY, maturity_boundary, "maturity boundary", BatchError)
    mesh = _method(exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times)
    return _grouped("fo_price_lsm_batch_f64", None, initial_spots, strikes, maturities, rates, volatilities,
                    _cash(dividend_offsets, dividend_times, dividend_amounts, 1, dividend_policy=policy,
                          maturity_boundary=boundary),
                    mesh, executor, training_paths, evaluation_paths, training_seed, training_domain_start,
                    evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit,
                    tie_rule, insufficient_exercise_support)


def price_lsm_call_batch_escrowed_cash_dividends_f64(  # noqa: PLR0913
    initial_spots, strikes, maturities, rates, volatilities, dividend_offsets, dividend_times, dividend_amounts,
    volatility_convention, maturity_boundary, exercise_mesh, base_intervals, origin_exercise,
    explicit_exercise_offsets, explicit_exercise_times, executor, training_paths, evaluation_paths, training_seed,
    training_domain_start, evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance,
    condition_limit, tie_rule, insufficient_exercise_support,
) -> tuple:
    convention = _parse(_ESCROWED_VOL, volatility_convention, "escrowed volatility convention")
    boundary = _parse(_MATURITY, maturity_boundary, "maturity boundary", BatchError)
    mesh = _method(exercise_mesh, base_intervals, origin_exercise, explicit_exercise_offsets, explicit_exercise_times)
    return _grouped("fo_price_lsm_batch_f64", None, initial_spots, strikes, maturities, rates, volatilities,
                    _cash(dividend_offsets, dividend_times, dividend_amounts, 2, volatility_convention=convention,
                          maturity_boundary=boundary),
                    mesh, executor, training_paths, evaluation_paths, training_seed, training_domain_start,
                    evaluation_seed, evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit,
                    tie_rule, insufficient_exercise_support)


def price_lsm_call_ragged_f64(  # noqa: PLR0913 - one argument per ragged column
    initial_spots, strikes, maturities, rates, volatilities, dividend_yields, dividend_offsets, dividend_times,
    dividend_amounts, dividend_policy, maturity_boundary, exercise_offsets, exercise_times, origin_exercise,
    training_paths, evaluation_paths, executor, training_seed, training_domain_start, evaluation_seed,
    evaluation_domain_start, polynomial_degree, rank_tolerance, condition_limit, tie_rule,
    insufficient_exercise_support, log_discount_nodes=None,
) -> tuple:
    """Ragged batch (per-contract path counts; no reference counterpart): NativeBatchLsmResult, and
    with log_discount_nodes (mesh nodes per row) also (delta, vega, dP/dL, offsets, dP/dD). With
    executor None the request is only validated (nothing is priced; returns None)."""
    handle = None if executor is None else _executor_handle(executor)
    request = lsm_ragged_request(
        initial_spots=initial_spots, strikes=strikes, maturities=maturities, rates=rates, volatilities=volatilities,
        dividend_yields=dividend_yields, dividend_offsets=dividend_offsets, dividend_times=dividend_times,
        dividend_amounts=dividend_amounts, dividend_policy=_parse(_DIVIDEND_POLICIES, dividend_policy, "dividend policy"),
        maturity_boundary=_parse(_MATURITY, maturity_boundary, "maturity boundary", BatchError),
        exercise_offsets=exercise_offsets, exercise_times=exercise_times,
        origin_exercise=_parse(_ORIGIN, origin_exercise, "origin exercise convention"),
        training_paths=training_paths, evaluation_paths=evaluation_paths, training_seed=training_seed,
        training_domain_start=training_domain_start, evaluation_seed=evaluation_seed,
        evaluation_domain_start=evaluation_domain_start, polynomial_degree=polynomial_degree,
        rank_tolerance=rank_tolerance, condition_limit=condition_limit,
        tie_rule=_parse(_TIE_RULES, tie_rule, "exercise tie rule"),
        insufficient_exercise_support=_parse(_SUPPORT, insufficient_exercise_support,
                                             "insufficient exercise support policy"),
    )
    err = _abi.FoError()
    if handle is None:
        _check(_lib().fo_validate_lsm_ragged_f64(ctypes.byref(request.struct), ctypes.byref(err)), err)
        return None
    columns = batch_columns(request.rows)
    greeks = None
    if log_discount_nodes is not None:
        rows = request.rows
        arrays = {"delta": np.zeros(rows), "vega": np.zeros(rows), "d_l": np.zeros(max(int(log_discount_nodes), 1)),
                  "offsets": np.zeros(rows + 1, dtype=np.int64),
                  "d_d": np.zeros(max(0 if dividend_times is None else int(dividend_times.size), 1))}
        greeks = _abi.FoRaggedGreeksColumns()
        greeks.delta = _dp(arrays["delta"])
        greeks.vega = _dp(arrays["vega"])
        greeks.log_discount_sensitivities = _dp(arrays["d_l"])
        greeks.log_discount_capacity = int(log_discount_nodes)
        greeks.log_discount_offsets = _ip(arrays["offsets"])
        greeks.dividend_sensitivities = _dp(arrays["d_d"])
    status = _lib().fo_price_lsm_ragged_f64(handle, ctypes.byref(request.struct), ctypes.byref(columns.struct),
                                            None if greeks is None else ctypes.byref(greeks), ctypes.byref(err))
    _check(status, err)
    if greeks is None:
        return columns.as_tuple()
    n_events = 0 if dividend_times is None else int(dividend_times.size)
    return (columns.as_tuple(), arrays["delta"], arrays["vega"], arrays["d_l"][: int(log_discount_nodes)],
            arrays["offsets"], arrays["d_d"][:n_events])
