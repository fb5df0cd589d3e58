"""Ragged batches (fo_price_lsm_ragged_f64): independent contracts with their own path counts.

Row r of a ragged batch is the contract of price_lsm_call on the union mesh of its exercise and
cash-dividend times with domains start + r; it is checked against the oracle's single-contract
restatement of the reference (prices / SD / SE within 1e-9 relative, stopping counts identical).
"""

from __future__ import annotations

import ctypes

import _oracle
import numpy as np
import pytest
from _workloads import ragged_columns, ragged_request, ragged_row_as_call
from finoptions import _abi
from finoptions._requests import batch_columns, lsm_call_request

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def gpu_ragged(native_executor, req):
    cols = batch_columns(req.rows)
    err = _abi.FoError()
    status = _abi.load().fo_price_lsm_ragged_f64(native_executor.raw, ctypes.byref(req.struct),
                                                 ctypes.byref(cols.struct), None, ctypes.byref(err))
    return status, err, (cols.as_tuple() if status == 0 else None)


def test_ragged_rows_match_single_contract_oracle_prices(native_executor) -> None:
    c = ragged_columns(16, seed=41, min_paths=1024, max_paths=16384, min_exercise=4, max_exercise=30)
    status, err, out = gpu_ragged(native_executor, ragged_request(c))
    assert status == 0, err.message
    for r in range(c.rows):
        want = _oracle.price_lsm_call(lsm_call_request(**ragged_row_as_call(c, r)), 8)
        price, _, sd, se, _, counts, diags = want
        assert out[0][r] == pytest.approx(price, rel=RTOL, abs=1e-13), r
        assert out[1][r] == pytest.approx(sd, rel=RTOL, abs=1e-13), r
        assert out[2][r] == pytest.approx(se, rel=RTOL, abs=1e-13), r
        assert out[10][r] == sum(counts[:-1]) and out[11][r] == counts[-1], r
        assert out[5][r] == sum(1 for d in diags if d[1] == "regression"), r


def test_rows_above_64ki_paths_match_the_oracle(native_executor) -> None:
    """Rows above 65,536 training paths are fitted by a cluster of four CTAs (the rest by one CTA
    each, in a concurrent launch); both kinds of row must still price like the single contract."""
    c = ragged_columns(6, seed=67, min_paths=40000, max_paths=140000, min_exercise=4, max_exercise=8)
    assert (c.paths > 65536).any() and (c.paths <= 65536).any()
    status, err, out = gpu_ragged(native_executor, ragged_request(c))
    assert status == 0, err.message
    for r in range(c.rows):
        want = _oracle.price_lsm_call(lsm_call_request(**ragged_row_as_call(c, r)), 8)
        price, _, sd, se, _, counts, diags = want
        assert out[0][r] == pytest.approx(price, rel=RTOL, abs=1e-13), r
        assert out[1][r] == pytest.approx(sd, rel=RTOL, abs=1e-13), r
        assert out[2][r] == pytest.approx(se, rel=RTOL, abs=1e-13), r
        assert out[10][r] == sum(counts[:-1]) and out[11][r] == counts[-1], r
        assert out[5][r] == sum(1 for d in diags if d[1] == "regression"), r


def _row(c, r: int):
    one = ragged_columns(1, seed=1, min_paths=2, max_paths=3, min_exercise=4, max_exercise=4)
    for name in ("initial_spots", "strikes", "maturities", "rates", "volatilities", "dividend_yields", "paths"):
        setattr(one, name, getattr(c, name)[r:r + 1].copy())
    one.exercise_times = c.exercise_times[c.exercise_offsets[r]:c.exercise_offsets[r + 1]].copy()
    one.exercise_offsets = np.array([0, one.exercise_times.size], dtype=np.int64)
    one.dividend_times = c.dividend_times[c.dividend_offsets[r]:c.dividend_offsets[r + 1]].copy()
    one.dividend_amounts = c.dividend_amounts[c.dividend_offsets[r]:c.dividend_offsets[r + 1]].copy()
    one.dividend_offsets = np.array([0, one.dividend_times.size], dtype=np.int64)
    return one


def test_ragged_row_equals_the_contract_priced_alone(native_executor) -> None:
    """A ragged row and the same contract alone (domains shifted to the row's) agree bit for bit."""
    c = ragged_columns(6, seed=43, min_paths=2048, max_paths=8192, min_exercise=4, max_exercise=20)
    status, err, out = gpu_ragged(native_executor, ragged_request(c))
    assert status == 0, err.message
    for r in (1, 4):
        status, err, single = gpu_ragged(native_executor, ragged_request(_row(c, r), training_domain_start=r,
                                                                         evaluation_domain_start=(1 << 20) + r))
        assert status == 0, err.message
        for column, values in zip(out, single, strict=True):
            assert column[r] == values[0]


def test_ragged_validation_reports_the_row(native_executor) -> None:
    c = ragged_columns(4, seed=47, min_paths=256, max_paths=512, min_exercise=4, max_exercise=6)
    c.paths[2] = 1
    status, err, _ = gpu_ragged(native_executor, ragged_request(c))
    assert status == _abi.FO_ERR_INPUT
    assert err.message.decode() == "batched LSM evaluation path count 1 at row 2 is outside [2, 4294967295]"


def gpu_ragged_greeks(native_executor, req, c):
    nodes = [len(ragged_row_as_call(c, r)["schedule_times"]) for r in range(c.rows)]
    g = _abi.FoRaggedGreeksColumns()
    delta, vega = np.zeros(c.rows), np.zeros(c.rows)
    d_l, offsets = np.zeros(sum(nodes)), np.zeros(c.rows + 1, dtype=np.int64)
    d_d = np.zeros(max(c.dividend_times.size, 1))
    g.delta = delta.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    g.vega = vega.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    g.log_discount_sensitivities = d_l.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    g.log_discount_capacity = d_l.size
    g.log_discount_offsets = offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    g.dividend_sensitivities = d_d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    cols = batch_columns(req.rows)
    err = _abi.FoError()
    status = _abi.load().fo_price_lsm_ragged_f64(native_executor.raw, ctypes.byref(req.struct),
                                                 ctypes.byref(cols.struct), ctypes.byref(g), ctypes.byref(err))
    assert status == 0, err.message
    assert offsets.tolist() == [0, *np.cumsum(nodes).tolist()]
    return cols.as_tuple(), delta, vega, d_l, offsets, d_d


@pytest.mark.parametrize("degree", [4, 1])
def test_ragged_greeks_match_the_single_contract_greeks(native_executor, degree) -> None:
    from finoptions._requests import lsm_call_greeks, lsm_call_result

    c = ragged_columns(10, seed=53, min_paths=2048, max_paths=16384, min_exercise=4, max_exercise=24)
    out, delta, vega, d_l, offsets, d_d = gpu_ragged_greeks(native_executor, ragged_request(c, degree=degree), c)
    _, _, plain = gpu_ragged(native_executor, ragged_request(c, degree=degree))
    np.testing.assert_allclose(out[0], plain[0], rtol=1e-13, atol=1e-14)
    for r in range(c.rows):
        kw = ragged_row_as_call(c, r, degree=degree)
        req = lsm_call_request(**kw)
        res = lsm_call_result(req.exercise_rows)
        n_div = len(kw["dividend_nodes"])
        g, g_l, g_d = lsm_call_greeks(len(kw["schedule_times"]), n_div)
        err = _abi.FoError()
        assert _abi.load().fo_price_lsm_call_greeks_f64(native_executor.raw, ctypes.byref(req.struct),
                                                        ctypes.byref(res.struct), ctypes.byref(g),
                                                        ctypes.byref(err)) == 0, err.message
        assert out[0][r] == pytest.approx(res.as_tuple()[0], rel=1e-12, abs=1e-13), r
        scale = max(abs(g.delta), 1.0)
        assert delta[r] == pytest.approx(g.delta, rel=1e-10, abs=1e-12 * scale), r
        assert vega[r] == pytest.approx(g.vega, rel=1e-10, abs=1e-10), r
        np.testing.assert_allclose(d_l[offsets[r]:offsets[r + 1]], g_l, rtol=1e-9, atol=1e-10, err_msg=str(r))
        first = int(c.dividend_offsets[r])
        np.testing.assert_allclose(d_d[first:first + n_div], g_d, rtol=1e-9, atol=1e-10, err_msg=str(r))


def test_public_ragged_api_matches_the_c_abi(executor, native_executor) -> None:
    import finoptions as fo

    c = ragged_columns(6, seed=59, min_paths=1024, max_paths=4096, min_exercise=4, max_exercise=12)
    contracts = fo.LsmRaggedContracts(
        initial_spots=c.initial_spots, strikes=c.strikes, maturities=c.maturities, rates=c.rates,
        volatilities=c.volatilities, exercise=fo.RaggedExerciseTimes(offsets=c.exercise_offsets, times=c.exercise_times),
        training_paths=c.paths, evaluation_paths=c.paths, dividend_yields=c.dividend_yields,
        cash_dividends=fo.RaggedCashDividends(offsets=c.dividend_offsets, times=c.dividend_times,
                                              amounts=c.dividend_amounts))
    kwargs = dict(contracts=contracts, origin_exercise=fo.OriginExercise.EXCLUDED, executor=executor,
                  training_stream=fo.RandomStream(seed=41, domain=0), evaluation_stream=fo.RandomStream(seed=41, domain=1 << 20),
                  insufficient_exercise_support=fo.InsufficientExerciseSupportPolicy.CONTINUE)
    prices = fo.price_lsm_call_ragged(**kwargs)
    result, greeks = fo.price_lsm_call_ragged_greeks(**kwargs)
    out, delta, vega, d_l, offsets, d_d = gpu_ragged_greeks(native_executor, ragged_request(c), c)
    _, _, plain = gpu_ragged(native_executor, ragged_request(c))
    np.testing.assert_array_equal(prices.prices, plain[0])
    np.testing.assert_array_equal(result.prices, out[0])
    np.testing.assert_array_equal(greeks.delta, delta)
    np.testing.assert_array_equal(greeks.log_discount_sensitivities, d_l)
    np.testing.assert_array_equal(greeks.log_discount_offsets, offsets)
    np.testing.assert_array_equal(greeks.dividend_sensitivities, d_d[:c.dividend_times.size])
    assert not greeks.delta.flags.writeable and not result.prices.flags.writeable
