"""Marshalling between Python values and the C ABI's request/result structs."""

from __future__ import annotations

import ctypes
import struct
from array import array
from collections.abc import Sequence
from dataclasses import dataclass
from itertools import chain
from typing import Any

import numpy as np

from . import _abi


def _f64(values: Sequence[float] | np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(values, dtype=np.float64)


def _u32(values: Sequence[int] | np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(values, dtype=np.uint32)


def _ptr(array: np.ndarray | None, ctype: type) -> Any:
    if array is None:
        return ctypes.POINTER(ctype)()
    return array.ctypes.data_as(ctypes.POINTER(ctype))


@dataclass
class CallRequest:
    """A filled FoLsmCallRequest and the arrays its pointers borrow."""

    struct: _abi.FoLsmCallRequest
    keepalive: tuple[Any, ...]
    exercise_rows: int


def _spans(parts: tuple[Any, ...], typecode: str, convert: Any) -> tuple[tuple[Any, ...], list[tuple[int, int]]]:
    """The buffers that hold `parts` and each part's (address, length) in them.

    Plain lists and tuples of numbers go into one array.array, back to back (one C-level
    conversion instead of a numpy conversion per part). Anything else, including elements that
    array.array refuses, is converted part by part with `convert`, so its errors are unchanged.
    """
    if all(type(p) is list or type(p) is tuple for p in parts):
        try:
            flat = array(typecode, chain.from_iterable(parts))
        except (TypeError, OverflowError, ValueError):
            pass
        else:
            base, step, spans = flat.buffer_info()[0], flat.itemsize, []
            for p in parts:
                spans.append((base, len(p)))
                base += step * len(p)
            return (flat,), spans
    arrays = tuple(convert(p) for p in parts)
    return arrays, [(a.ctypes.data, a.size) for a in arrays]


def lsm_call_request(
    *,
    initial_spot: float,
    strike: float,
    schedule_times: Sequence[float],
    curve_times: Sequence[float],
    log_discounts: Sequence[float],
    dividend_yield_times: Sequence[float],
    cumulative_dividend_yields: Sequence[float],
    dividend_nodes: Sequence[int],
    dividend_amounts: Sequence[float],
    exercise_nodes: Sequence[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: int,
    training_paths: int,
    evaluation_paths: int,
    training_seed: int,
    training_domain: int,
    evaluation_seed: int,
    evaluation_domain: int,
    polynomial_degree: int,
    rank_tolerance: float,
    condition_limit: float,
    tie_rule: int,
    insufficient_exercise_support: int,
) -> CallRequest:
    floats, (st, ct, ld, yt, cy, da) = _spans(
        (schedule_times, curve_times, log_discounts, dividend_yield_times, cumulative_dividend_yields,
         dividend_amounts), "d", _f64)
    nodes, (dn, en) = _spans((dividend_nodes, exercise_nodes), "I", _u32)
    q = _abi.FoLsmCallRequest()
    q.initial_spot = initial_spot
    q.strike = strike
    q.schedule_times, q.n_schedule_times = st
    q.curve_times, q.n_curve_times = ct
    q.log_discounts, q.n_log_discounts = ld
    q.dividend_yield_times, q.n_dividend_yield_times = yt
    q.cumulative_dividend_yields, q.n_cumulative_dividend_yields = cy
    q.dividend_nodes, q.n_dividend_nodes = dn
    q.dividend_amounts, q.n_dividend_amounts = da
    q.exercise_nodes, q.n_exercise_nodes = en
    q.expiry_node = expiry_node
    q.annualized_volatility = annualized_volatility
    q.dividend_policy = dividend_policy
    q.training_paths = training_paths
    q.evaluation_paths = evaluation_paths
    q.training_seed = training_seed
    q.training_domain = training_domain
    q.evaluation_seed = evaluation_seed
    q.evaluation_domain = evaluation_domain
    q.polynomial_degree = polynomial_degree
    q.rank_tolerance = rank_tolerance
    q.condition_limit = condition_limit
    q.tie_rule = tie_rule
    q.insufficient_exercise_support = insufficient_exercise_support
    return CallRequest(q, floats + nodes, en[1])


def _record_format(structure: type) -> struct.Struct:
    """A little-endian struct.Struct that reads `structure` (a ctypes.Structure of scalar fields)
    field by field, with the padding its ctypes offsets imply."""
    codes = {ctypes.c_uint32: "I", ctypes.c_int32: "i", ctypes.c_uint64: "Q", ctypes.c_int64: "q",
             ctypes.c_double: "d"}
    fmt, at = "<", 0
    for name, ctype in structure._fields_:
        offset = getattr(structure, name).offset
        fmt += f"{offset - at}x" if offset > at else ""
        fmt += codes[ctype]
        at = offset + ctypes.sizeof(ctype)
    size = ctypes.sizeof(structure)
    fmt += f"{size - at}x" if size > at else ""
    packed = struct.Struct(fmt)
    if packed.size != size:  # pragma: no cover - the layout is fixed by the C header
        msg = f"{structure.__name__}: format {fmt} reads {packed.size} bytes of {size}"
        raise ImportError(msg)
    return packed


_DIAGNOSTIC = _record_format(_abi.FoLsmNodeDiagnostic)
if array("d").itemsize != 8 or array("I").itemsize != 4:  # pragma: no cover - every supported platform
    msg = "array.array('d'/'I') must be binary64 / 32-bit to back the C ABI's double / uint32_t arrays"
    raise ImportError(msg)


@dataclass
class CallResult:
    """Caller-owned result buffers for one single-contract call."""

    struct: _abi.FoLsmCallResult
    observation_nodes: np.ndarray
    exercise_counts: np.ndarray
    diagnostics: ctypes.Array

    def head(self) -> tuple:
        """(price, paths, sample SD or None, SE or None, observation nodes, exercise counts)."""
        r = self.struct
        rows = r.n_observations
        return (
            r.price,
            r.paths,
            r.sample_standard_deviation if r.has_sample_standard_deviation else None,
            r.standard_error if r.has_standard_error else None,
            self.observation_nodes[:rows].tolist(),
            self.exercise_counts[:rows].tolist(),
        )

    def rows(self) -> list[tuple]:
        """The diagnostics as plain tuples (node, kind code, exercise, estimated continuation,
        in-the-money paths, observations, columns, rank, condition, predictor mean, scale)."""
        n = self.struct.n_diagnostics
        if n > len(self.diagnostics):
            msg = f"native result reports {n} diagnostics for a buffer of {len(self.diagnostics)}"
            raise ValueError(msg)
        return list(_DIAGNOSTIC.iter_unpack(memoryview(self.diagnostics).cast("B")[: n * _DIAGNOSTIC.size]))

    def as_tuple(self) -> tuple:
        """NativeLsmResult-shaped tuple (crates/finoptions-python/src/lib.rs:1074-1082)."""
        diags = []
        for (node, kind, exercise, continuation, itm, observations, columns, rank, condition, mean,
             scale) in self.rows():
            if kind == _abi.FO_DIAG_ORIGIN_DECISION:
                diags.append((node, "origin_decision", bool(exercise), continuation, None, None, None, None,
                              None, None, None))
            elif kind == _abi.FO_DIAG_NO_IN_THE_MONEY_PATHS:
                diags.append((node, "no_in_the_money_paths", None, None, None, None, None, None, None, None,
                              None))
            elif kind == _abi.FO_DIAG_INSUFFICIENT_SUPPORT:
                diags.append((node, "insufficient_exercise_support", None, None, itm, None, columns, None,
                              None, None, None))
            else:
                diags.append((node, "regression", None, None, itm, observations, columns, rank, condition, mean,
                              scale))
        return (*self.head(), diags)


def lsm_call_result(exercise_rows: int) -> CallResult:
    rows = exercise_rows + 1
    columns = np.zeros(2 * rows, dtype=np.uint32)
    diags = (_abi.FoLsmNodeDiagnostic * max(exercise_rows, 1))()
    r = _abi.FoLsmCallResult()
    r.observation_nodes = columns.ctypes.data
    r.observation_capacity = rows
    r.exercise_counts = r.observation_nodes + 4 * rows
    r.diagnostics = ctypes.addressof(diags)
    r.diagnostics_capacity = exercise_rows
    return CallResult(r, columns[:rows], columns[rows:], diags)


def lsm_call_greeks(nodes: int, dividends: int) -> tuple[_abi.FoLsmCallGreeks, np.ndarray, np.ndarray]:
    """An fo_lsm_call_greeks with caller-owned sensitivity buffers (keep the arrays alive)."""
    d_log_discounts = np.zeros(max(nodes, 1))
    d_dividends = np.zeros(max(dividends, 1))
    g = _abi.FoLsmCallGreeks()
    g.log_discount_sensitivities = _ptr(d_log_discounts, ctypes.c_double)
    g.log_discount_capacity = nodes
    g.dividend_sensitivities = _ptr(d_dividends, ctypes.c_double)
    g.dividend_capacity = dividends
    return g, d_log_discounts[:nodes], d_dividends[:dividends]


@dataclass
class RaggedRequest:
    struct: _abi.FoLsmRaggedRequest
    keepalive: tuple[Any, ...]
    rows: int


def lsm_ragged_request(
    *,
    initial_spots: np.ndarray,
    strikes: np.ndarray,
    maturities: np.ndarray,
    rates: np.ndarray,
    volatilities: np.ndarray,
    dividend_yields: np.ndarray | None,
    dividend_offsets: np.ndarray | None,
    dividend_times: np.ndarray | None,
    dividend_amounts: np.ndarray | None,
    dividend_policy: int,
    maturity_boundary: int,
    exercise_offsets: np.ndarray,
    exercise_times: np.ndarray,
    origin_exercise: int,
    training_paths: np.ndarray,
    evaluation_paths: np.ndarray,
    training_seed: int,
    training_domain_start: int,
    evaluation_seed: int,
    evaluation_domain_start: int,
    polynomial_degree: int,
    rank_tolerance: float,
    condition_limit: float,
    tie_rule: int,
    insufficient_exercise_support: int,
) -> RaggedRequest:
    q = _abi.FoLsmRaggedRequest()
    keep = (initial_spots, strikes, maturities, rates, volatilities, dividend_yields, dividend_offsets, dividend_times,
            dividend_amounts, exercise_offsets, exercise_times, training_paths, evaluation_paths)
    q.rows = int(initial_spots.size)
    q.initial_spots = _ptr(initial_spots, ctypes.c_double)
    q.strikes = _ptr(strikes, ctypes.c_double)
    q.maturities = _ptr(maturities, ctypes.c_double)
    q.rates = _ptr(rates, ctypes.c_double)
    q.volatilities = _ptr(volatilities, ctypes.c_double)
    q.dividend_yields = _ptr(dividend_yields, ctypes.c_double)
    q.dividend_offsets = _ptr(dividend_offsets, ctypes.c_int64)
    q.n_dividend_offsets = 0 if dividend_offsets is None else int(dividend_offsets.size)
    q.dividend_times = _ptr(dividend_times, ctypes.c_double)
    q.dividend_amounts = _ptr(dividend_amounts, ctypes.c_double)
    q.n_dividend_events = 0 if dividend_times is None else int(dividend_times.size)
    q.dividend_policy = dividend_policy
    q.maturity_boundary = maturity_boundary
    q.exercise_offsets = _ptr(exercise_offsets, ctypes.c_int64)
    q.n_exercise_offsets = int(exercise_offsets.size)
    q.exercise_times = _ptr(exercise_times, ctypes.c_double)
    q.n_exercise_times = int(exercise_times.size)
    q.origin_exercise = origin_exercise
    q.training_paths = _ptr(training_paths, ctypes.c_uint64)
    q.evaluation_paths = _ptr(evaluation_paths, ctypes.c_uint64)
    q.training_seed = training_seed
    q.training_domain_start = training_domain_start
    q.evaluation_seed = evaluation_seed
    q.evaluation_domain_start = evaluation_domain_start
    q.polynomial_degree = polynomial_degree
    q.rank_tolerance = rank_tolerance
    q.condition_limit = condition_limit
    q.tie_rule = tie_rule
    q.insufficient_exercise_support = insufficient_exercise_support
    return RaggedRequest(q, keep, q.rows)


@dataclass
class GroupedRequest:
    struct: _abi.FoLsmGroupedRequest
    keepalive: tuple[Any, ...]
    rows: int


def lsm_grouped_request(
    *,
    group_offsets: np.ndarray | None,
    initial_spots: np.ndarray,
    strikes: np.ndarray,
    maturities: np.ndarray,
    rates: np.ndarray,
    volatilities: np.ndarray,
    dividend_model: int,
    dividend_yields: np.ndarray | None = None,
    dividend_offsets: np.ndarray | None = None,
    dividend_times: np.ndarray | None = None,
    dividend_amounts: np.ndarray | None = None,
    dividend_policy: int = 0,
    maturity_boundary: int = 0,
    volatility_convention: int = 0,
    exercise_mesh: int,
    base_intervals: int | None,
    origin_exercise: int | None,
    explicit_exercise_offsets: np.ndarray | None,
    explicit_exercise_times: np.ndarray | None,
    training_paths: int,
    evaluation_paths: int,
    training_seed: int,
    training_domain_start: int,
    evaluation_seed: int,
    evaluation_domain_start: int,
    polynomial_degree: int,
    rank_tolerance: float,
    condition_limit: float,
    tie_rule: int,
    insufficient_exercise_support: int,
) -> GroupedRequest:
    q = _abi.FoLsmGroupedRequest()
    keep: list[Any] = []

    def put(name: str, array: np.ndarray | None, ctype: type) -> None:
        keep.append(array)
        setattr(q, name, _ptr(array, ctype))
        setattr(q, "n_" + name, 0 if array is None else int(array.size))

    put("group_offsets", group_offsets, ctypes.c_uint32)
    put("initial_spots", initial_spots, ctypes.c_double)
    put("strikes", strikes, ctypes.c_double)
    put("maturities", maturities, ctypes.c_double)
    put("rates", rates, ctypes.c_double)
    put("volatilities", volatilities, ctypes.c_double)
    q.dividend_model = dividend_model
    put("dividend_yields", dividend_yields, ctypes.c_double)
    put("dividend_offsets", dividend_offsets, ctypes.c_int64)
    put("dividend_times", dividend_times, ctypes.c_double)
    put("dividend_amounts", dividend_amounts, ctypes.c_double)
    q.dividend_policy = dividend_policy
    q.maturity_boundary = maturity_boundary
    q.volatility_convention = volatility_convention
    q.exercise_mesh = exercise_mesh
    q.has_base_intervals = 0 if base_intervals is None else 1
    q.base_intervals = 0 if base_intervals is None else base_intervals
    q.has_origin_exercise = 0 if origin_exercise is None else 1
    q.origin_exercise = 0 if origin_exercise is None else origin_exercise
    put("explicit_exercise_offsets", explicit_exercise_offsets, ctypes.c_int64)
    put("explicit_exercise_times", explicit_exercise_times, ctypes.c_double)
    q.training_paths = training_paths
    q.evaluation_paths = evaluation_paths
    q.training_seed = training_seed
    q.training_domain_start = training_domain_start
    q.evaluation_seed = evaluation_seed
    q.evaluation_domain_start = evaluation_domain_start
    q.polynomial_degree = polynomial_degree
    q.rank_tolerance = rank_tolerance
    q.condition_limit = condition_limit
    q.tie_rule = tie_rule
    q.insufficient_exercise_support = insufficient_exercise_support
    return GroupedRequest(q, tuple(keep), int(strikes.size))


@dataclass
class BatchColumns:
    struct: _abi.FoBatchResultColumns
    arrays: dict[str, np.ndarray]

    def as_tuple(self) -> tuple[np.ndarray, ...]:
        a = self.arrays
        return (
            a["prices"], a["sample_standard_deviations"], a["standard_errors"],
            a["origin_decisions_fitted"].astype(np.bool_), a["origin_exercised"].astype(np.bool_),
            a["regression_nodes"], a["no_training_support_nodes"],
            a["insufficient_exercise_support_nodes"], a["minimum_in_the_money_training_paths"],
            a["maximum_regression_condition_numbers"], a["early_exercise_paths"], a["expiry_paths"],
        )


_COLUMN_TYPES = (
    ("prices", np.float64, ctypes.c_double),
    ("sample_standard_deviations", np.float64, ctypes.c_double),
    ("standard_errors", np.float64, ctypes.c_double),
    ("origin_decisions_fitted", np.uint8, ctypes.c_uint8),
    ("origin_exercised", np.uint8, ctypes.c_uint8),
    ("regression_nodes", np.uint32, ctypes.c_uint32),
    ("no_training_support_nodes", np.uint32, ctypes.c_uint32),
    ("insufficient_exercise_support_nodes", np.uint32, ctypes.c_uint32),
    ("minimum_in_the_money_training_paths", np.uint32, ctypes.c_uint32),
    ("maximum_regression_condition_numbers", np.float64, ctypes.c_double),
    ("early_exercise_paths", np.uint32, ctypes.c_uint32),
    ("expiry_paths", np.uint32, ctypes.c_uint32),
)


def batch_columns(rows: int) -> BatchColumns:
    s = _abi.FoBatchResultColumns()
    s.rows = rows
    arrays: dict[str, np.ndarray] = {}
    for name, dtype, ctype in _COLUMN_TYPES:
        array = np.zeros(rows, dtype=dtype)
        arrays[name] = array
        setattr(s, name, _ptr(array, ctype))
    return BatchColumns(s, arrays)


@dataclass
class GbmRequest:
    struct: _abi.FoGbmSeededRequest
    keepalive: tuple[np.ndarray, ...]
    rows: int


def gbm_seeded_request(
    *,
    initial_spot: float,
    schedule_times: Sequence[float],
    curve_times: Sequence[float],
    log_discounts: Sequence[float],
    dividend_yield_times: Sequence[float],
    cumulative_dividend_yields: Sequence[float],
    dividend_nodes: Sequence[int],
    dividend_amounts: Sequence[float],
    exercise_nodes: Sequence[int],
    expiry_node: int,
    annualized_volatility: float,
    dividend_policy: int,
    paths: int,
    seed: int,
    domain: int,
) -> GbmRequest:
    arrays = (
        _f64(schedule_times), _f64(curve_times), _f64(log_discounts), _f64(dividend_yield_times),
        _f64(cumulative_dividend_yields), _u32(dividend_nodes), _f64(dividend_amounts), _u32(exercise_nodes),
    )
    st, ct, ld, yt, cy, dn, da, en = arrays
    q = _abi.FoGbmSeededRequest()
    q.initial_spot = initial_spot
    q.schedule_times, q.n_schedule_times = _ptr(st, ctypes.c_double), st.size
    q.curve_times, q.n_curve_times = _ptr(ct, ctypes.c_double), ct.size
    q.log_discounts, q.n_log_discounts = _ptr(ld, ctypes.c_double), ld.size
    q.dividend_yield_times, q.n_dividend_yield_times = _ptr(yt, ctypes.c_double), yt.size
    q.cumulative_dividend_yields, q.n_cumulative_dividend_yields = _ptr(cy, ctypes.c_double), cy.size
    q.dividend_nodes, q.n_dividend_nodes = _ptr(dn, ctypes.c_uint32), dn.size
    q.dividend_amounts, q.n_dividend_amounts = _ptr(da, ctypes.c_double), da.size
    q.exercise_nodes, q.n_exercise_nodes = _ptr(en, ctypes.c_uint32), en.size
    q.expiry_node = expiry_node
    q.annualized_volatility = annualized_volatility
    q.dividend_policy = dividend_policy
    q.paths = paths
    q.seed = seed
    q.domain = domain
    return GbmRequest(q, arrays, int(en.size) + 1)
