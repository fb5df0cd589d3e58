"""Parity on the benchmark workloads' own inputs, at their full sizes.

* The weekly single contract at 2^20 + 2^20 paths: price, SD and SE against the oracle, and the
  decision-flip count - evaluation paths whose stopping row differs between the engine and the
  oracle, path by path - which must be zero. The engine's regression sums run in a different order
  than the reference's sequential ones (and its GBM step uses CUDA's exp), so its fitted
  coefficients differ from the oracle's in the last bits; a path flips only if its exercise value
  falls within that difference of the fitted continuation value.
* The ragged workload (1,024 contracts, seed 41): the rows with the most paths (up to 262,144) and
  the most exercise dates (up to 104), plus a seeded random sample, against the oracle's single
  contract prices.
* The grouped workload (4,096 states x 8 strikes at 32,768 + 32,768 paths, seed 23): the full call
  on the device, and a sample of its states - the widest meshes, the most dividends, and a seeded
  random sample - against the oracle's grouped restatement of those states.
"""

from __future__ import annotations

import ctypes
import os

import _oracle
import numpy as np
import pytest
from _workloads import (
    EVALUATION_DOMAIN_START,
    TRAINING_DOMAIN_START,
    grouped_columns,
    grouped_request,
    ragged_columns,
    ragged_request,
    ragged_row_as_call,
    weekly_call_kwargs,
)
from finoptions import _abi
from finoptions._requests import batch_columns, lsm_call_request, lsm_call_result
from test_gpu_batch import assert_columns, gpu_batch

pytestmark = pytest.mark.gpu

RTOL = 1e-9
THREADS = max(1, min(32, os.cpu_count() or 1))


def test_weekly_contract_at_full_size_has_no_decision_flips(native_executor) -> None:
    kwargs = weekly_call_kwargs(1 << 20)
    req = lsm_call_request(**kwargs)
    lib, err = _abi.load(), _abi.FoError()
    plan = ctypes.c_void_p()
    assert lib.fo_lsm_call_plan_create(native_executor.raw, ctypes.byref(req.struct), ctypes.byref(plan),
                                       ctypes.byref(err)) == 0, err.message
    try:
        assert lib.fo_lsm_call_plan_launch(plan, ctypes.byref(err)) == 0, err.message
        res = lsm_call_result(req.exercise_rows)
        assert lib.fo_lsm_call_plan_collect(plan, ctypes.byref(res.struct), ctypes.byref(err)) == 0, err.message
        gpu = res.as_tuple()
        gpu_stops = np.zeros(1 << 20, dtype=np.uint32)
        assert lib.fo_lsm_call_plan_stopping_rows(plan, gpu_stops.ctypes.data, gpu_stops.size,
                                                  ctypes.byref(err)) == 0, err.message
    finally:
        lib.fo_lsm_call_plan_destroy(plan)
    prices, _, oracle_stops = _oracle.price_markets(req, [req], refit=True, threads=THREADS)
    flips = int((gpu_stops != oracle_stops[0]).sum())
    print(f"\n[bench-rows] weekly 2^20: price {gpu[0]!r} oracle {prices[0]!r}, decision flips {flips}")
    assert flips == 0
    assert gpu[0] == pytest.approx(prices[0], rel=RTOL)
    assert tuple(int(v) for v in np.bincount(oracle_stops[0], minlength=req.exercise_rows + 1)) == tuple(gpu[5])


def _ragged_sample(c, each: int = 4, seed: int = 7) -> list[int]:
    n_ex = np.diff(c.exercise_offsets)
    by_paths = np.argsort(-c.paths.astype(np.int64), kind="stable")[:each]
    by_dates = np.argsort(-n_ex, kind="stable")[:each]
    rng = np.random.Generator(np.random.PCG64(seed))
    rest = rng.choice(c.rows, size=each, replace=False)
    return sorted({int(r) for r in (*by_paths, *by_dates, *rest)})


def test_benchmark_ragged_rows_match_the_oracle(native_executor) -> None:
    c = ragged_columns(1024, seed=41)
    req = ragged_request(c)
    cols = batch_columns(req.rows)
    err = _abi.FoError()
    assert _abi.load().fo_price_lsm_ragged_f64(native_executor.raw, ctypes.byref(req.struct), ctypes.byref(cols.struct),
                                               None, ctypes.byref(err)) == 0, err.message
    out = cols.as_tuple()
    rows = _ragged_sample(c)
    assert int(c.paths.max()) in {int(c.paths[r]) for r in rows}
    assert int(np.diff(c.exercise_offsets).max()) in {int(np.diff(c.exercise_offsets)[r]) for r in rows}
    for r in rows:
        price, _, sd, se, _, counts, diags = _oracle.price_lsm_call(lsm_call_request(**ragged_row_as_call(c, r)),
                                                                    THREADS)
        assert out[0][r] == pytest.approx(price, rel=RTOL, abs=1e-13), r
        assert out[1][r] == pytest.approx(sd, rel=RTOL, abs=1e-13), r
        assert out[2][r] == pytest.approx(se, rel=RTOL, abs=1e-13), r
        assert out[10][r] == sum(counts[:-1]) and out[11][r] == counts[-1], r
        assert out[5][r] == sum(1 for d in diags if d[1] == "regression"), r


def _state(c, g: int):
    """State g of a grouped workload as a one-group workload (the same populations: its domains are
    moved to start + g)."""
    one = grouped_columns(1, 8, seed=1)
    for name in ("initial_spots", "maturities", "rates", "volatilities"):
        setattr(one, name, getattr(c, name)[g:g + 1].copy())
    k = int(c.group_offsets[1] - c.group_offsets[0])
    one.strikes = c.strikes[g * k:(g + 1) * k].copy()
    one.group_offsets = np.array([0, k], dtype=np.uint32)
    one.exercise_times = c.exercise_times[c.exercise_offsets[g]:c.exercise_offsets[g + 1]].copy()
    one.exercise_offsets = np.array([0, one.exercise_times.size], dtype=np.int64)
    one.dividend_times = c.dividend_times[c.dividend_offsets[g]:c.dividend_offsets[g + 1]].copy()
    one.dividend_amounts = c.dividend_amounts[c.dividend_offsets[g]:c.dividend_offsets[g + 1]].copy()
    one.dividend_offsets = np.array([0, one.dividend_times.size], dtype=np.int64)
    return one


def test_benchmark_grouped_states_match_the_oracle(native_executor) -> None:
    paths = 1 << 15
    c = grouped_columns(4096, 8, seed=23)
    status, err, out = gpu_batch(native_executor, grouped_request(c, paths))
    assert status == 0, err.message
    n_ex, n_div = np.diff(c.exercise_offsets), np.diff(c.dividend_offsets)
    rng = np.random.Generator(np.random.PCG64(11))
    states = sorted({*np.argsort(-n_ex, kind="stable")[:4].tolist(), *np.argsort(-n_div, kind="stable")[:4].tolist(),
                     *rng.choice(c.groups, size=8, replace=False).tolist()})
    for g in states:
        one = _state(c, g)
        req = grouped_request(one, paths)
        req.struct.training_domain_start = TRAINING_DOMAIN_START + g
        req.struct.evaluation_domain_start = EVALUATION_DOMAIN_START + g
        want = _oracle.price_lsm_grouped(req, THREADS)
        assert_columns(tuple(col[8 * g:8 * (g + 1)] for col in out), want)
