"""Load the CPU parity oracle (oracle/_build/liboracle.so) for the test suite.

The oracle is test infrastructure: a C++ restatement of the reference path that the tests use as
the checker. It is built from oracle/ by `make` when missing.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np
from finoptions import _abi
from finoptions._requests import (
    CallRequest,
    GbmRequest,
    GroupedRequest,
    batch_columns,
    lsm_call_result,
)

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "liboracle.so"

_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    global _lib  # noqa: PLW0603 - one oracle handle per process
    if _lib is None:
        if not ORACLE_LIB.is_file():
            subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, capture_output=True)
        lib = ctypes.CDLL(str(ORACLE_LIB))
        err = ctypes.POINTER(_abi.FoError)
        lib.orc_sample_normals.argtypes = [
            ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
        ]
        lib.orc_normal_after_budget.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        lib.orc_moments.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint64, ctypes.c_void_p]
        lib.orc_recurrence_moments.argtypes = [ctypes.c_void_p] * 5 + [
            ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
        ]
        lib.orc_apply_dividend.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double]
        lib.orc_apply_dividend.restype = ctypes.c_double
        lib.orc_fit_regression.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
            ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
        ]
        lib.orc_predict.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        lib.orc_simulate_gbm_seeded.argtypes = [
            ctypes.POINTER(_abi.FoGbmSeededRequest), ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64, err,
        ]
        lib.orc_simulate_gbm.argtypes = [
            ctypes.POINTER(_abi.FoGbmSeededRequest), ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64,
            err,
        ]
        lib.orc_price_lsm_call.argtypes = [
            ctypes.POINTER(_abi.FoLsmCallRequest), ctypes.c_int32, ctypes.POINTER(_abi.FoLsmCallResult), err,
            ctypes.POINTER(ctypes.c_int32),
        ]
        lib.orc_price_lsm_call_markets.argtypes = [
            ctypes.POINTER(_abi.FoLsmCallRequest), ctypes.POINTER(_abi.FoLsmCallRequest), ctypes.c_uint64,
            ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, err,
        ]
        lib.orc_price_lsm_grouped.argtypes = [
            ctypes.POINTER(_abi.FoLsmGroupedRequest), ctypes.c_int32, ctypes.POINTER(_abi.FoBatchResultColumns), err,
        ]
        lib.orc_exact_union_times.argtypes = [
            ctypes.c_double, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
        ]
        lib.orc_exact_union_times.restype = ctypes.c_uint64
        lib.orc_exact_explicit_union_times.argtypes = [
            ctypes.c_double, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
            ctypes.c_uint64,
        ]
        lib.orc_exact_explicit_union_times.restype = ctypes.c_uint64
        _lib = lib
    return _lib


class OracleFailure(Exception):
    """The oracle reported a typed failure (code, stage, error record)."""

    def __init__(self, status: int, error: _abi.FoError, stage: int = 0) -> None:
        super().__init__(error.message.decode())
        self.status = status
        self.code = error.code
        self.row = error.row
        self.group = error.group
        self.node = error.node
        self.path = error.path
        self.stage = stage


def normals(seed: int, domain: int, path_start: int, paths: int, count: int) -> np.ndarray:
    out = np.zeros((paths, count))
    status = load().orc_sample_normals(seed, domain, path_start, paths, count, out.ctypes.data)
    if status:
        raise OracleFailure(status, _abi.FoError())
    return out


def simulate(request: GbmRequest, threads: int = 8) -> np.ndarray:
    q = request.struct
    out = np.zeros((request.rows, int(q.paths)))
    err = _abi.FoError()
    status = load().orc_simulate_gbm_seeded(ctypes.byref(q), threads, out.ctypes.data, out.size, ctypes.byref(err))
    if status:
        raise OracleFailure(status, err)
    return out


def simulate_from(request: GbmRequest, normals: np.ndarray, threads: int = 8) -> np.ndarray:
    """States [rows, paths] stepped by the caller's normals [intervals, paths] (simulate_gbm_f64)."""
    q = request.struct
    normals = np.ascontiguousarray(normals, dtype=np.float64)
    out = np.zeros((request.rows, int(q.paths)))
    err = _abi.FoError()
    status = load().orc_simulate_gbm(ctypes.byref(q), normals.ctypes.data, threads, out.ctypes.data, out.size,
                                     ctypes.byref(err))
    if status:
        raise OracleFailure(status, err)
    return out


def price_lsm_call(request: CallRequest, threads: int = 8) -> tuple:
    result = lsm_call_result(request.exercise_rows)
    err = _abi.FoError()
    stage = ctypes.c_int32(0)
    status = load().orc_price_lsm_call(
        ctypes.byref(request.struct), threads, ctypes.byref(result.struct), ctypes.byref(err), ctypes.byref(stage)
    )
    if status:
        raise OracleFailure(status, err, stage.value)
    return result.as_tuple()


def price_markets(base: CallRequest, markets: list[CallRequest], *, refit: bool, threads: int = 8,
                  paths: bool = True, frozen_stops: np.ndarray | None = None
                  ) -> tuple[np.ndarray, np.ndarray | None, np.ndarray | None]:
    """One contract on several markets with common random numbers: refit=True prices each market
    from scratch (the reference's bump-and-reprice), refit=False evaluates every market with the
    policy fitted once on `base`, or, given frozen_stops, stops path p at row frozen_stops[p] in
    every market. Returns prices [markets] and, with paths=True, every path's discounted payoff and
    stopping row [markets, evaluation paths]."""
    n = len(markets)
    table = (_abi.FoLsmCallRequest * n)(*[m.struct for m in markets])
    prices = np.zeros(n)
    n_paths = int(base.struct.evaluation_paths)
    payoffs = np.zeros((n, n_paths)) if paths else None
    stops = np.zeros((n, n_paths), dtype=np.uint32) if paths else None
    err = _abi.FoError()
    frozen = None
    if frozen_stops is not None:
        frozen = np.ascontiguousarray(frozen_stops, dtype=np.uint32)
        assert frozen.size == n_paths
    status = load().orc_price_lsm_call_markets(
        ctypes.byref(base.struct), table, n, 1 if refit else 0, None if frozen is None else frozen.ctypes.data,
        threads, prices.ctypes.data,
        payoffs.ctypes.data if paths else None, stops.ctypes.data if paths else None, ctypes.byref(err))
    if status:
        raise OracleFailure(status, err)
    return prices, payoffs, stops


def price_lsm_grouped(request: GroupedRequest, threads: int = 8) -> tuple:
    columns = batch_columns(request.rows)
    err = _abi.FoError()
    status = load().orc_price_lsm_grouped(ctypes.byref(request.struct), threads, ctypes.byref(columns.struct),
                                          ctypes.byref(err))
    if status:
        raise OracleFailure(status, err)
    return columns.as_tuple()


def fit_regression(x: np.ndarray, y: np.ndarray, degree: int, rank_tolerance: float = 1e-12,
                   condition_limit: float = 1e8) -> tuple[int, np.ndarray, tuple[int, int]]:
    model = np.zeros(22)
    aux = np.zeros(2, dtype=np.int64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    code = load().orc_fit_regression(x.ctypes.data, y.ctypes.data, x.size, degree, rank_tolerance,
                                     condition_limit, model.ctypes.data, aux.ctypes.data)
    return int(code), model, (int(aux[0]), int(aux[1]))


def predict(model: np.ndarray, degree: int, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(x.size)
    code = load().orc_predict(model.ctypes.data, degree, x.ctypes.data, x.size, out.ctypes.data)
    assert code == 0
    return out
