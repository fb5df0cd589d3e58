"""Grouped and row-addressed batches on the B200 against the oracle (pricing.rs:191-589).

Every test calls the C ABI (fo_price_lsm_grouped_f64 / fo_price_lsm_batch_f64) or the public
Python API over it, and compares all twelve row-result columns with the oracle's restatement of
the reference on the same seeded inputs: prices, standard deviations and errors within 1e-9
relative, counts and flags identical, condition numbers within 1e-6 relative (they come from the
fitted design, whose last bits differ between the two regression algorithms).
"""

from __future__ import annotations

import ctypes

import _oracle
import numpy as np
import pytest
from _workloads import GroupedColumns, grouped_columns, grouped_request
from finoptions import _abi
from finoptions._requests import batch_columns, lsm_call_request, lsm_call_result, lsm_grouped_request
from test_gpu_parity import ORACLE_CODES, _abi_code

pytestmark = pytest.mark.gpu

RTOL = 1e-9
COLUMNS = ("prices", "sample_standard_deviations", "standard_errors", "origin_decisions_fitted", "origin_exercised",
           "regression_nodes", "no_training_support_nodes", "insufficient_exercise_support_nodes",
           "minimum_in_the_money_training_paths", "maximum_regression_condition_numbers", "early_exercise_paths",
           "expiry_paths")


def gpu_batch(native_executor, req, grouped: bool = True):
    columns = batch_columns(req.rows)
    err = _abi.FoError()
    fn = _abi.load().fo_price_lsm_grouped_f64 if grouped else _abi.load().fo_price_lsm_batch_f64
    status = fn(native_executor.raw, ctypes.byref(req.struct), ctypes.byref(columns.struct), ctypes.byref(err))
    return status, err, (columns.as_tuple() if status == 0 else None)


def assert_columns(got: tuple, want: tuple) -> None:
    for name, g, w in zip(COLUMNS, got, want, strict=True):
        if name in ("prices", "sample_standard_deviations", "standard_errors"):
            np.testing.assert_allclose(g, w, rtol=RTOL, atol=1e-13, err_msg=name)
        elif name == "maximum_regression_condition_numbers":
            np.testing.assert_allclose(g, w, rtol=1e-6, err_msg=name)
        else:
            np.testing.assert_array_equal(g, w, err_msg=name)


def check_against_oracle(native_executor, req, grouped: bool = True) -> tuple | None:
    status, err, gpu = gpu_batch(native_executor, req, grouped)
    try:
        want = _oracle.price_lsm_grouped(req, 16)
    except _oracle.OracleFailure as failure:
        assert status != 0, "the oracle failed but the device priced the batch"
        assert err.code == _abi_code(ORACLE_CODES[failure.code]), err.message
        assert err.row == failure.row, err.message
        return None
    assert status == 0, err.message
    assert_columns(gpu, want)
    return gpu


def row_columns(c: GroupedColumns) -> GroupedColumns:
    """The grouped columns expanded to one contract per row (each row repeats its group's market)."""
    per = np.diff(c.group_offsets.astype(np.int64))
    rep = lambda a: np.repeat(a, per)  # noqa: E731
    ex = [c.exercise_times[c.exercise_offsets[g]:c.exercise_offsets[g + 1]] for g in range(c.groups)]
    dv = [(c.dividend_times[c.dividend_offsets[g]:c.dividend_offsets[g + 1]],
           c.dividend_amounts[c.dividend_offsets[g]:c.dividend_offsets[g + 1]]) for g in range(c.groups)]
    ex_rows = [ex[g] for g in range(c.groups) for _ in range(per[g])]
    dv_rows = [dv[g] for g in range(c.groups) for _ in range(per[g])]
    offsets = lambda parts: np.concatenate([[0], np.cumsum([p.size for p in parts])]).astype(np.int64)  # noqa: E731
    return GroupedColumns(
        group_offsets=np.arange(c.rows + 1, dtype=np.uint32),
        initial_spots=rep(c.initial_spots), strikes=c.strikes.copy(), maturities=rep(c.maturities),
        rates=rep(c.rates), volatilities=rep(c.volatilities),
        dividend_offsets=offsets([d[0] for d in dv_rows]),
        dividend_times=np.concatenate([d[0] for d in dv_rows]) if dv_rows else np.zeros(0),
        dividend_amounts=np.concatenate([d[1] for d in dv_rows]) if dv_rows else np.zeros(0),
        exercise_offsets=offsets(ex_rows), exercise_times=np.concatenate(ex_rows),
    )


def test_grouped_cash_dividends_on_explicit_meshes_match_the_oracle(native_executor) -> None:
    c = grouped_columns(12, strikes_per_group=4, seed=5, min_exercise=6, max_exercise=20)
    out = check_against_oracle(native_executor, grouped_request(c, 4096))
    assert out is not None
    assert (out[10].astype(np.int64) + out[11] == 4096).all()


def test_grouped_with_the_origin_decision_matches_the_oracle(native_executor) -> None:
    c = grouped_columns(8, strikes_per_group=8, seed=9, min_exercise=4, max_exercise=12)
    out = check_against_oracle(native_executor, grouped_request(c, 2048, origin=1))
    assert out is not None and out[3].all()


def test_grouped_fail_policy_matches_the_oracle_or_fails_identically(native_executor) -> None:
    c = grouped_columns(16, strikes_per_group=8, seed=13, min_exercise=6, max_exercise=16)
    check_against_oracle(native_executor, grouped_request(c, 1024, support=0))


@pytest.mark.parametrize("degree", [0, 1, 3])
def test_grouped_lower_degrees_match_the_oracle(native_executor, degree) -> None:
    """Each regression degree runs its own instance of the batch backward and evaluation kernels."""
    c = grouped_columns(8, strikes_per_group=5, seed=61 + degree, min_exercise=6, max_exercise=14)
    assert check_against_oracle(native_executor, grouped_request(c, 2048, degree=degree)) is not None


def test_grouped_tiny_populations_raise_the_oracle_error(native_executor) -> None:
    """With 8 training paths some strike has 1..4 in-the-money paths at a row: the fail policy
    raises InsufficientObservations for the lowest failing row."""
    c = grouped_columns(6, strikes_per_group=4, seed=3, min_exercise=6, max_exercise=10)
    req = grouped_request(c, 8, support=0, degree=4)
    status, err, _ = gpu_batch(native_executor, req)
    with pytest.raises(_oracle.OracleFailure) as failure:
        _oracle.price_lsm_grouped(req, 4)
    assert status == _abi.FO_ERR_LSM
    assert err.code == _abi_code(ORACLE_CODES[failure.value.code])
    assert err.row == failure.value.row
    assert err.message.decode().startswith(f"LSM batch estimator failed at row {failure.value.row}: ")


def test_grouped_escrowed_spot_matched_volatility_matches_the_oracle(native_executor) -> None:
    c = grouped_columns(10, strikes_per_group=3, seed=17, min_exercise=6, max_exercise=18)
    check_against_oracle(native_executor, grouped_request(c, 4096, dividend_model=2, volatility_convention=1))


def test_grouped_escrowed_prepaid_forward_matches_the_oracle(native_executor) -> None:
    c = grouped_columns(10, strikes_per_group=3, seed=19, min_exercise=6, max_exercise=18)
    check_against_oracle(native_executor, grouped_request(c, 4096, dividend_model=2, volatility_convention=0))


def test_grouped_continuous_yield_on_a_uniform_mesh_matches_the_oracle(native_executor) -> None:
    rng = np.random.Generator(np.random.PCG64(29))
    groups, per = 9, 5
    spots = rng.uniform(60, 140, groups)
    req = lsm_grouped_request(
        group_offsets=(np.arange(groups + 1) * per).astype(np.uint32), initial_spots=spots,
        strikes=(spots[:, None] * np.linspace(0.85, 1.15, per)).reshape(-1).copy(),
        maturities=rng.uniform(0.3, 1.5, groups), rates=rng.uniform(0.0, 0.06, groups),
        volatilities=rng.uniform(0.15, 0.5, groups), dividend_model=0,
        dividend_yields=rng.uniform(0.0, 0.05, groups), exercise_mesh=0, base_intervals=16, origin_exercise=1,
        explicit_exercise_offsets=None, explicit_exercise_times=None, training_paths=4096, evaluation_paths=4096,
        training_seed=7, training_domain_start=100, evaluation_seed=7, evaluation_domain_start=200,
        polynomial_degree=3, rank_tolerance=1e-12, condition_limit=1e8, tie_rule=1, insufficient_exercise_support=1,
    )
    check_against_oracle(native_executor, req)


def test_grouped_cash_dividend_date_mesh_matches_the_oracle(native_executor) -> None:
    c = grouped_columns(10, strikes_per_group=4, seed=31, min_exercise=6, max_exercise=18)
    keep = np.diff(c.dividend_offsets) > 0  # the cash-date mesh needs at least one dividend to exercise
    req = lsm_grouped_request(
        group_offsets=c.group_offsets, initial_spots=c.initial_spots, strikes=c.strikes, maturities=c.maturities,
        rates=c.rates, volatilities=c.volatilities, dividend_model=1, dividend_offsets=c.dividend_offsets,
        dividend_times=c.dividend_times, dividend_amounts=c.dividend_amounts, dividend_policy=1,
        maturity_boundary=0, exercise_mesh=1, base_intervals=None, origin_exercise=None,
        explicit_exercise_offsets=None, explicit_exercise_times=None, training_paths=2048, evaluation_paths=2048,
        training_seed=3, training_domain_start=0, evaluation_seed=4, evaluation_domain_start=50,
        polynomial_degree=2, rank_tolerance=1e-12, condition_limit=1e8, tie_rule=0, insufficient_exercise_support=1,
    )
    assert keep.any()
    check_against_oracle(native_executor, req)


def test_row_batch_matches_the_oracle_and_one_strike_groups_bitwise(native_executor) -> None:
    c = row_columns(grouped_columns(5, strikes_per_group=3, seed=37, min_exercise=5, max_exercise=14))
    rows = check_against_oracle(native_executor, grouped_request(c, 2048, grouped=False), grouped=False)
    status, err, groups = gpu_batch(native_executor, grouped_request(c, 2048, grouped=True), grouped=True)
    assert status == 0, err.message
    assert rows is not None
    for name, a, b in zip(COLUMNS, rows, groups, strict=True):
        np.testing.assert_array_equal(a, b, err_msg=name)


def test_one_row_batch_matches_the_scalar_entry(native_executor) -> None:
    """A one-contract row batch prices the contract of price_lsm_call on the same union mesh."""
    c = row_columns(grouped_columns(1, strikes_per_group=1, seed=41, min_exercise=10, max_exercise=10))
    status, err, batch = gpu_batch(native_executor, grouped_request(c, 8192, grouped=False), grouped=False)
    assert status == 0, err.message
    T, r = float(c.maturities[0]), float(c.rates[0])
    ex, cash = c.exercise_times, c.dividend_times
    times = [0.0, *np.union1d(ex, cash).tolist(), T]
    nodes = {t: i for i, t in enumerate(times)}
    req = lsm_call_request(
        initial_spot=float(c.initial_spots[0]), strike=float(c.strikes[0]), schedule_times=times, curve_times=times,
        log_discounts=[0.0 if i == 0 else -r * t for i, t in enumerate(times)], dividend_yield_times=times,
        cumulative_dividend_yields=[0.0] * len(times), dividend_nodes=[nodes[t] for t in cash.tolist()],
        dividend_amounts=c.dividend_amounts.tolist(), exercise_nodes=[nodes[t] for t in ex.tolist()],
        expiry_node=len(times) - 1, annualized_volatility=float(c.volatilities[0]), dividend_policy=0,
        training_paths=8192, evaluation_paths=8192, training_seed=23, training_domain=0, evaluation_seed=23,
        evaluation_domain=1 << 20, polynomial_degree=4, rank_tolerance=1e-12, condition_limit=1e8, tie_rule=0,
        insufficient_exercise_support=1,
    )
    result = lsm_call_result(req.exercise_rows)
    assert _abi.load().fo_price_lsm_call_f64(native_executor.raw, ctypes.byref(req.struct), ctypes.byref(result.struct),
                                             ctypes.byref(err)) == 0, err.message
    price, paths, sd, se, _, counts, _ = result.as_tuple()
    np.testing.assert_allclose([batch[0][0], batch[1][0], batch[2][0]], [price, sd, se], rtol=1e-12)
    assert batch[10][0] == sum(counts[:-1]) and batch[11][0] == counts[-1]


def test_cfg3_shaped_groups_match_the_oracle(native_executor) -> None:
    """48 states x 8 strikes at 32,768 + 32,768 paths per state (the benchmark's shapes)."""
    c = grouped_columns(48, strikes_per_group=8, seed=23)
    check_against_oracle(native_executor, grouped_request(c, 32768))


def test_public_grouped_api_returns_frozen_columns(executor, native_executor) -> None:
    import finoptions as fo

    c = grouped_columns(4, strikes_per_group=3, seed=43, min_exercise=5, max_exercise=9)
    groups = fo.LsmStrikeGroups(
        group_offsets=c.group_offsets, initial_spots=c.initial_spots, strikes=c.strikes, maturities=c.maturities,
        rates=c.rates, volatilities=c.volatilities,
        dividends=fo.CashDividendBatch(
            schedules=fo.RaggedCashDividends(offsets=c.dividend_offsets, times=c.dividend_times,
                                             amounts=c.dividend_amounts),
            policy=fo.DividendPolicy.LIQUIDATOR, maturity_boundary=fo.MaturityBoundary.STRICTLY_BEFORE),
    )
    mesh = fo.ExplicitExerciseMesh(schedules=fo.RaggedExerciseTimes(offsets=c.exercise_offsets, times=c.exercise_times),
                                   origin_exercise=fo.OriginExercise.EXCLUDED)
    method = fo.Lsm(training_paths=2048, evaluation_paths=2048, training_stream=fo.RandomStream(seed=23, domain=0),
                    evaluation_stream=fo.RandomStream(seed=23, domain=1 << 20),
                    insufficient_exercise_support=fo.InsufficientExerciseSupportPolicy.CONTINUE)
    result = fo.price_lsm_call_grouped_batch(groups=groups, mesh=mesh, executor=executor, method=method)
    assert not result.prices.flags.writeable
    status, err, raw = gpu_batch(native_executor, grouped_request(c, 2048))
    assert status == 0, err.message
    np.testing.assert_array_equal(result.prices, raw[0])
    np.testing.assert_array_equal(result.expiry_paths, raw[11])


@pytest.mark.parametrize(
    ("mutate", "message"),
    [
        (lambda c: c.group_offsets.__setitem__(0, 1), "LSM grouped batch offsets must start at zero; observed 1"),
        (lambda c: c.strikes.__setitem__(3, -1.0), "LSM batch field strikes is invalid at row 3: observed -1.0"),
        (lambda c: c.volatilities.__setitem__(1, 0.0),
         "LSM batch field constant_volatilities is invalid at row 1: observed 0.0"),
    ],
)
def test_grouped_validation_messages(native_executor, mutate, message) -> None:
    c = grouped_columns(3, strikes_per_group=2, seed=47, min_exercise=4, max_exercise=6)
    mutate(c)
    status, err, _ = gpu_batch(native_executor, grouped_request(c, 256))
    assert status == _abi.FO_ERR_INPUT
    assert err.message.decode() == message


def test_overlapping_domain_ranges_are_rejected(native_executor) -> None:
    c = grouped_columns(3, strikes_per_group=2, seed=47, min_exercise=4, max_exercise=6)
    req = grouped_request(c, 256)
    req.struct.evaluation_domain_start = 2
    status, err, _ = gpu_batch(native_executor, req)
    assert status == _abi.FO_ERR_INPUT
    assert err.message.decode() == "batched LSM training domains [0, 3) overlap evaluation domains [2, 5)"


def test_arrow_tables_price_like_the_numpy_columns(executor) -> None:
    """The same grouped request from pyarrow tables (finoptions.arrow) and from NumPy columns."""
    import finoptions as fo
    import pyarrow as pa
    from finoptions import arrow

    c = grouped_columns(6, strikes_per_group=4, seed=47, min_exercise=5, max_exercise=12)
    mesh = fo.ExplicitExerciseMesh(schedules=fo.RaggedExerciseTimes(offsets=c.exercise_offsets, times=c.exercise_times),
                                   origin_exercise=fo.OriginExercise.EXCLUDED)
    method = fo.Lsm(training_paths=4096, evaluation_paths=4096, training_stream=fo.RandomStream(seed=23, domain=0),
                    evaluation_stream=fo.RandomStream(seed=23, domain=1 << 20),
                    insufficient_exercise_support=fo.InsufficientExerciseSupportPolicy.CONTINUE)
    div = [c.dividend_times[c.dividend_offsets[g]:c.dividend_offsets[g + 1]].tolist() for g in range(c.groups)]
    amt = [c.dividend_amounts[c.dividend_offsets[g]:c.dividend_offsets[g + 1]].tolist() for g in range(c.groups)]
    states = pa.table({"spot": c.initial_spots, "maturity": c.maturities, "rate": c.rates, "vol": c.volatilities,
                       "div_times": pa.array(div, type=pa.large_list(pa.float64())),
                       "div_amounts": pa.array(amt, type=pa.large_list(pa.float64()))})
    strikes = pa.table({"strike": c.strikes})
    table = arrow.price_lsm_strike_group_tables(
        states, strikes, group_offsets=pa.array(c.group_offsets, type=pa.uint32()),
        state_columns=arrow.LsmStrikeGroupColumns(initial_spot="spot", maturity="maturity", rate="rate",
                                                  volatility="vol"),
        strike_column="strike",
        dividends=arrow.CashDividendColumns(times="div_times", amounts="div_amounts",
                                            policy=fo.DividendPolicy.LIQUIDATOR,
                                            maturity_boundary=fo.MaturityBoundary.STRICTLY_BEFORE),
        mesh=mesh, executor=executor, method=method)
    groups = fo.LsmStrikeGroups(
        group_offsets=c.group_offsets, initial_spots=c.initial_spots, strikes=c.strikes, maturities=c.maturities,
        rates=c.rates, volatilities=c.volatilities,
        dividends=fo.CashDividendBatch(
            schedules=fo.RaggedCashDividends(offsets=c.dividend_offsets, times=c.dividend_times,
                                             amounts=c.dividend_amounts),
            policy=fo.DividendPolicy.LIQUIDATOR, maturity_boundary=fo.MaturityBoundary.STRICTLY_BEFORE))
    direct = fo.price_lsm_call_grouped_batch(groups=groups, mesh=mesh, executor=executor, method=method)
    assert table.num_rows == c.strikes.size
    for name in ("prices", "standard_errors", "early_exercise_paths", "maximum_regression_condition_numbers"):
        np.testing.assert_array_equal(table.column(name).to_numpy(), getattr(direct, name), err_msg=name)
