"""Marshalling of the single-contract request and result (finoptions._requests), on the CPU.

The request packs plain lists into one binary64 and one uint32 buffer and gives the C ABI
addresses into them; every field must read back as the per-array conversion would have written
it, and inputs that the packed path refuses must fail exactly as before.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from finoptions import _abi
from finoptions._requests import _f64, _spans, _u32, lsm_call_request, lsm_call_result

ARRAYS = (("schedule_times", "n_schedule_times", ctypes.c_double),
          ("curve_times", "n_curve_times", ctypes.c_double),
          ("log_discounts", "n_log_discounts", ctypes.c_double),
          ("dividend_yield_times", "n_dividend_yield_times", ctypes.c_double),
          ("cumulative_dividend_yields", "n_cumulative_dividend_yields", ctypes.c_double),
          ("dividend_nodes", "n_dividend_nodes", ctypes.c_uint32),
          ("dividend_amounts", "n_dividend_amounts", ctypes.c_double),
          ("exercise_nodes", "n_exercise_nodes", ctypes.c_uint32))


def request_kwargs(**overrides) -> dict:
    kw = dict(
        initial_spot=100.0, strike=95.0, schedule_times=[0.0, 0.25, 0.5, 1.0], curve_times=[0.0, 0.5, 1.0],
        log_discounts=[0.0, -0.02, -0.04], dividend_yield_times=[0.0, 1.0], cumulative_dividend_yields=[0.0, 0.01],
        dividend_nodes=[2], dividend_amounts=[1.5], exercise_nodes=[0, 1, 2], expiry_node=3,
        annualized_volatility=0.2, dividend_policy=0, training_paths=64, evaluation_paths=64, training_seed=1,
        training_domain=2, evaluation_seed=3, evaluation_domain=4, polynomial_degree=2, rank_tolerance=1e-12,
        condition_limit=1e8, tie_rule=0, insufficient_exercise_support=0)
    kw.update(overrides)
    return kw


def read_back(struct: _abi.FoLsmCallRequest) -> dict:
    out = {}
    for field, length, ctype in ARRAYS:
        n = getattr(struct, length)
        address = getattr(struct, field)
        out[field] = list((ctype * n).from_address(address)) if n else []
    return out


@pytest.mark.parametrize("container", [list, tuple])
def test_packed_request_reads_back_every_array(container) -> None:
    kw = request_kwargs()
    packed = {k: container(v) if isinstance(v, list) else v for k, v in kw.items()}
    request = lsm_call_request(**packed)
    got = read_back(request.struct)
    for field, _, _ in ARRAYS:
        assert got[field] == [float(v) for v in kw[field]] or got[field] == list(kw[field]), field
    assert request.exercise_rows == 3
    assert len(request.keepalive) == 2  # one binary64 and one uint32 buffer


def test_numpy_and_mixed_inputs_take_the_per_array_path() -> None:
    kw = request_kwargs(schedule_times=np.array([0.0, 0.25, 0.5, 1.0]), exercise_nodes=np.array([0, 1, 2]))
    request = lsm_call_request(**kw)
    got = read_back(request.struct)
    assert got["schedule_times"] == [0.0, 0.25, 0.5, 1.0]
    assert got["exercise_nodes"] == [0, 1, 2]
    assert got["curve_times"] == [0.0, 0.5, 1.0]
    assert len(request.keepalive) == 8


def test_empty_arrays_have_zero_length() -> None:
    request = lsm_call_request(**request_kwargs(dividend_nodes=[], dividend_amounts=[]))
    assert request.struct.n_dividend_nodes == 0 and request.struct.n_dividend_amounts == 0
    assert read_back(request.struct)["exercise_nodes"] == [0, 1, 2]


@pytest.mark.parametrize(("part", "dtype"), [(["1.5", 2.0], np.float64), ([[1.0, 2.0]], np.float64),
                                             ([-1, 2], np.uint32), ([1.5, 2], np.uint32)])
def test_refused_elements_fail_or_convert_as_numpy_does(part, dtype) -> None:
    typecode, convert = ("d", _f64) if dtype is np.float64 else ("I", _u32)
    try:
        expected = convert(part)
    except Exception as exc:  # noqa: BLE001 - the exception type itself is compared
        with pytest.raises(type(exc)):
            _spans((part,), typecode, convert)
        return
    buffers, spans = _spans((part,), typecode, convert)
    (address, n), = spans
    ctype = ctypes.c_double if dtype is np.float64 else ctypes.c_uint32
    assert n == expected.size
    assert list((ctype * n).from_address(address)) == expected.ravel().tolist()
    assert buffers[0] is not None


def test_result_reader_builds_the_native_result_shape() -> None:
    res = lsm_call_result(4)  # room for four diagnostics and five observation rows
    r = res.struct
    r.price, r.paths, r.has_sample_standard_deviation, r.sample_standard_deviation = 4.5, 64, 1, 2.0
    r.has_standard_error, r.standard_error = 0, 0.0
    r.n_observations, r.n_diagnostics = 4, 4
    nodes = (ctypes.c_uint32 * 4).from_address(r.observation_nodes)
    counts = (ctypes.c_uint32 * 4).from_address(r.exercise_counts)
    nodes[:] = [0, 1, 2, 3]
    counts[:] = [5, 6, 7, 8]
    d = res.diagnostics
    d[0].node, d[0].kind, d[0].exercise, d[0].estimated_continuation = 0, _abi.FO_DIAG_ORIGIN_DECISION, 1, 3.25
    d[1].node, d[1].kind = 1, _abi.FO_DIAG_NO_IN_THE_MONEY_PATHS
    d[2].node, d[2].kind, d[2].in_the_money_paths, d[2].columns = 2, _abi.FO_DIAG_INSUFFICIENT_SUPPORT, 2, 3
    d[3].node, d[3].kind, d[3].in_the_money_paths, d[3].observations = 3, _abi.FO_DIAG_REGRESSION, 40, 40
    d[3].columns, d[3].rank, d[3].condition_number, d[3].predictor_mean, d[3].predictor_scale = 3, 3, 12.5, 1.1, 0.2
    price, paths, sd, se, obs, cnt, diags = res.as_tuple()
    assert (price, paths, sd, se, obs, cnt) == (4.5, 64, 2.0, None, [0, 1, 2, 3], [5, 6, 7, 8])
    assert diags == [
        (0, "origin_decision", True, 3.25, None, None, None, None, None, None, None),
        (1, "no_in_the_money_paths", None, None, None, None, None, None, None, None, None),
        (2, "insufficient_exercise_support", None, None, 2, None, 3, None, None, None, None),
        (3, "regression", None, None, 40, 40, 3, 3, 12.5, 1.1, 0.2),
    ]
    assert all(type(v) is int for v in obs + cnt)


def test_records_built_from_rows_equal_the_records_of_the_native_tuples() -> None:
    from finoptions import lsm  # noqa: PLC0415 - the pricing module's private builders

    res = lsm_call_result(5)
    r = res.struct
    r.n_observations, r.n_diagnostics = 6, 5
    d = res.diagnostics
    d[0].node, d[0].kind, d[0].exercise, d[0].estimated_continuation = 0, _abi.FO_DIAG_ORIGIN_DECISION, 0, 1.75
    d[1].node, d[1].kind = 1, _abi.FO_DIAG_NO_IN_THE_MONEY_PATHS
    d[2].node, d[2].kind, d[2].in_the_money_paths, d[2].columns = 2, _abi.FO_DIAG_INSUFFICIENT_SUPPORT, 1, 5
    for i, kind in ((3, _abi.FO_DIAG_REGRESSION), (4, 7)):  # an unknown kind reads as a regression row
        d[i].node, d[i].kind, d[i].in_the_money_paths, d[i].observations, d[i].columns = i, kind, 90 + i, 90 + i, 5
        d[i].rank, d[i].condition_number, d[i].predictor_mean, d[i].predictor_scale = 5, 3.5 + i, 1.0 + i, 0.25
    expected = tuple(lsm._fit_diagnostic(row) for row in res.as_tuple()[6])
    got = lsm._fit_records(res.rows())
    assert got == expected
    assert [type(x).__name__ for x in got] == ["OriginDecisionDiagnostics", "NoInTheMoneyPathsDiagnostics",
                                               "InsufficientExerciseSupportDiagnostics",
                                               "RegressionFitDiagnostics", "RegressionFitDiagnostics"]


def test_diagnostic_rows_read_the_ctypes_layout() -> None:
    res = lsm_call_result(6)
    r = res.struct
    r.n_diagnostics = 6
    for i in range(6):
        d = res.diagnostics[i]
        d.node, d.kind, d.exercise, d.estimated_continuation = i, i % 4, i & 1, 0.5 * i
        d.in_the_money_paths, d.observations, d.columns, d.rank = 2**32 - 1 - i, 2**40 + i, 5, 4
        d.condition_number, d.predictor_mean, d.predictor_scale = 1e8 - i, -1.5 * i, 2.0**-i
    expected = np.frombuffer(res.diagnostics, dtype=np.dtype(_abi.FoLsmNodeDiagnostic), count=6).tolist()
    assert res.rows() == expected
    r.n_diagnostics = 7  # more than the buffer holds
    with pytest.raises(ValueError, match="7 diagnostics"):
        res.rows()
