"""GPU parity: the sm_100a kernels, through the C ABI, against the CPU oracle on the same inputs.

Bars (as the engine's contract states them):
  * Philox words / ZIGNOR normals: bit-exact;
  * path states: bit-exact except where CUDA's and glibc's exp differ by an ulp, so at least half
    of all states are bit-identical and every state agrees to 1e-13 relative;
  * price and standard error: 1e-9 relative; stopping counts, in-the-money counts, diagnostic
    kinds and ranks: identical; predictor mean / scale: 1e-12 relative; condition numbers 1e-8.
"""

from __future__ import annotations

import ctypes
import json
import math
from pathlib import Path

import numpy as np
import pytest
from finoptions import _abi
from finoptions._requests import gbm_seeded_request, lsm_call_request, lsm_call_result

import _oracle
from _workloads import grouped_columns, grouped_row_as_call

pytestmark = pytest.mark.gpu
GOLDEN = json.loads((Path(__file__).parent / "golden" / "golden.json").read_text())
PRICE_RTOL = 1e-9


def weekly(steps=52, maturity=1.0, rate=0.04, q=0.02, sigma=0.25, dividends=(), exercise=None, policy=0):
    t = [i * maturity / steps for i in range(steps + 1)]
    return dict(
        schedule_times=t, curve_times=t, log_discounts=[0.0 if i == 0 else -rate * t[i] for i in range(steps + 1)],
        dividend_yield_times=t, cumulative_dividend_yields=[0.0 if i == 0 else q * t[i] for i in range(steps + 1)],
        dividend_nodes=[d[0] for d in dividends], dividend_amounts=[d[1] for d in dividends],
        exercise_nodes=list(range(steps)) if exercise is None else exercise, expiry_node=steps,
        annualized_volatility=sigma, dividend_policy=policy,
    )


CFG1 = dict(schedule_times=[0.0, 0.5, 1.0], curve_times=[0.0, 0.5, 1.0], log_discounts=[0.0, -0.01, -0.025],
            dividend_yield_times=[0.0, 0.5, 1.0], cumulative_dividend_yields=[0.0, 0.0, 0.0], dividend_nodes=[1],
            dividend_amounts=[2.0], exercise_nodes=[1], expiry_node=2, annualized_volatility=0.2, dividend_policy=0)


def request(plan, *, S0=100.0, K=100.0, paths=8192, seeds=((11, 1), (11, 2)), degree=4, tie=0, support=0,
            eval_paths=None):
    (ts, td), (es, ed) = seeds
    return lsm_call_request(initial_spot=S0, strike=K, training_paths=paths,
                            evaluation_paths=paths if eval_paths is None else eval_paths, training_seed=ts,
                            training_domain=td, evaluation_seed=es, evaluation_domain=ed, polynomial_degree=degree,
                            rank_tolerance=1e-12, condition_limit=1e8, tie_rule=tie,
                            insufficient_exercise_support=support, **plan)


def gpu_price(native_executor, req):
    result = lsm_call_result(req.exercise_rows)
    err = _abi.FoError()
    status = _abi.load().fo_price_lsm_call_f64(native_executor.raw, ctypes.byref(req.struct),
                                               ctypes.byref(result.struct), ctypes.byref(err))
    return status, err, (result.as_tuple() if status == 0 else None)


def assert_parity(gpu, oracle):
    price, paths, sd, se, nodes, counts, diags = gpu
    o_price, o_paths, o_sd, o_se, o_nodes, o_counts, o_diags = oracle
    assert paths == o_paths and nodes == o_nodes
    assert counts == o_counts
    assert math.isclose(price, o_price, rel_tol=PRICE_RTOL, abs_tol=1e-300)
    if o_sd is None:
        assert sd is None and se is None
    else:
        assert math.isclose(sd, o_sd, rel_tol=PRICE_RTOL, abs_tol=1e-300)
        assert math.isclose(se, o_se, rel_tol=PRICE_RTOL, abs_tol=1e-300)
    assert len(diags) == len(o_diags)
    for d, o in zip(diags, o_diags, strict=True):
        assert d[:2] == o[:2]
        if d[1] == "regression":
            assert d[4:8] == o[4:8]  # itm, observations, columns, rank
            assert math.isclose(d[8], o[8], rel_tol=1e-8)
            assert math.isclose(d[9], o[9], rel_tol=1e-12)
            assert math.isclose(d[10], o[10], rel_tol=1e-12)
        elif d[1] == "origin_decision":
            assert d[2] == o[2]
            assert math.isclose(d[3], o[3], rel_tol=PRICE_RTOL)
        else:
            assert d == o


def test_zignor_pin_and_bulk_normals_are_bit_exact(native_executor) -> None:
    lib = _abi.load()
    z = GOLDEN["zignor"]
    out = np.zeros(z["count"])
    err = _abi.FoError()
    assert lib.fo_sample_standard_normals_f64(native_executor.raw, z["seed"], z["domain"], z["path"], 1, z["count"],
                                              out.ctypes.data_as(_abi.c_double_p), out.size, ctypes.byref(err)) == 0
    assert [int(b) for b in out.view(np.uint64)] == z["bits"]
    paths, count = 30000, 60
    gpu = np.zeros(paths * count)
    assert lib.fo_sample_standard_normals_f64(native_executor.raw, 0xDEADBEEF12345, 77, 1000, paths, count,
                                              gpu.ctypes.data_as(_abi.c_double_p), gpu.size, ctypes.byref(err)) == 0
    cpu = _oracle.normals(0xDEADBEEF12345, 77, 1000, paths, count).ravel()
    assert np.array_equal(gpu.view(np.uint64), cpu.view(np.uint64))


@pytest.mark.parametrize("policy", [0, 1])
def test_seeded_paths_match_the_oracle(native_executor, policy) -> None:
    plan = weekly(dividends=((13, 1.5), (39, 1.5), (52, 0.5)), policy=policy)
    req = gbm_seeded_request(initial_spot=100.0, paths=40000, seed=11, domain=1, **plan)
    gpu = np.zeros(req.rows * 40000)
    err = _abi.FoError()
    assert _abi.load().fo_simulate_gbm_seeded_f64(native_executor.raw, ctypes.byref(req.struct),
                                                  gpu.ctypes.data_as(_abi.c_double_p), gpu.size, ctypes.byref(err)) == 0
    cpu = _oracle.simulate(req).ravel()
    same = gpu.view(np.uint64) == cpu.view(np.uint64)
    assert same.mean() > 0.5
    assert np.max(np.abs(gpu - cpu) / np.maximum(np.abs(cpu), 1e-300)) <= 1e-13


SCENARIOS = {
    "cfg1_readme": (CFG1, dict(paths=65536, seeds=((7, 1), (7, 2)))),
    "weekly_yield": (weekly(), dict(paths=16384)),
    "weekly_cash_liquidator": (weekly(dividends=((13, 1.5), (39, 1.5))), dict(paths=16384)),
    "weekly_cash_survivor": (weekly(dividends=((13, 4.0), (39, 4.0)), policy=1), dict(paths=16384)),
    "terminal_cash": (weekly(steps=12, dividends=((6, 2.0), (12, 3.0))), dict(paths=8192)),
    "degree_0": (weekly(steps=12), dict(paths=8192, degree=0)),
    "degree_1": (weekly(steps=12), dict(paths=8192, degree=1)),
    "degree_2": (weekly(steps=12), dict(paths=8192, degree=2)),
    "degree_3": (weekly(steps=12), dict(paths=8192, degree=3)),
    "greater_or_equal": (weekly(steps=12), dict(paths=8192, tie=1)),
    "deep_itm": (weekly(), dict(paths=16384, K=70.0)),
    "otm_continue": (weekly(), dict(paths=16384, K=135.0, support=1)),
    "otm_fail": (weekly(), dict(paths=16384, K=135.0)),
    "origin_included": (weekly(steps=8, exercise=list(range(8))), dict(paths=8192, S0=130.0)),
    "sparse_exercise": (weekly(steps=20, exercise=[3, 9, 15]), dict(paths=8192)),
    "odd_paths": (weekly(steps=10), dict(paths=5003)),
    "uneven_roles": (weekly(steps=10), dict(paths=3001, eval_paths=7777)),
    "continue_small": (weekly(steps=6, q=0.1, rate=0.01), dict(paths=16, K=120.0, support=1)),
    "european": (weekly(steps=4, exercise=[]), dict(paths=4096)),
}


@pytest.mark.parametrize("name", sorted(SCENARIOS))
def test_price_lsm_call_matches_the_oracle(native_executor, name) -> None:
    plan, kw = SCENARIOS[name]
    req = request(plan, **kw)
    status, err, gpu = gpu_price(native_executor, req)
    try:
        oracle = _oracle.price_lsm_call(req, 16)
    except _oracle.OracleFailure as failure:
        # Both engines must raise the same typed failure at the same node.
        assert status == _abi.FO_ERR_LSM
        assert err.code == _abi_code(ORACLE_CODES[failure.code])
        assert err.node == failure.node
        return
    assert status == 0, err.message
    assert_parity(gpu, oracle)


ORACLE_CODES = {
    1: "FO_CODE_RANDOM_NORMAL_BUDGET_EXHAUSTED",
    2: "FO_CODE_RANDOM_NORMAL_REJECTION_LIMIT",
    3: "FO_CODE_NON_FINITE_PATH_TRANSITION",
    10: "FO_CODE_INSUFFICIENT_OBSERVATIONS",
    13: "FO_CODE_DEGENERATE_PREDICTOR",
    14: "FO_CODE_RANK_DEFICIENT",
    15: "FO_CODE_CONDITION_LIMIT_EXCEEDED",
    17: "FO_CODE_NON_FINITE_FIT",
    20: "FO_CODE_NON_FINITE_DISCOUNTED_PAYOFF",
    21: "FO_CODE_EVALUATION_OUTSIDE_TRAINING_SUPPORT",
}


def test_a_row_far_from_the_previous_rows_mean_is_fitted_about_its_own(native_executor) -> None:
    """Strike 1.2 S0 of a 17-date state (row 55 of the seed-71 grouped columns): its first exercise
    row has 6 in-the-money paths whose mean moneyness (1.0023, sd 0.0026) lies nine standard
    deviations from the next row's (1.026), the pivot its power sums are staged about. The engine
    takes that row's sums again about its own mean; its condition number and the price match the
    oracle."""
    c = grouped_columns(12, 8, seed=71, min_exercise=6, max_exercise=20)
    req = lsm_call_request(**grouped_row_as_call(c, 55, 4096))
    status, err, gpu = gpu_price(native_executor, req)
    assert status == 0, err.message
    oracle = _oracle.price_lsm_call(req, 16)
    assert_parity(gpu, oracle)
    assert gpu[6][0][4] == 6
    assert math.isclose(gpu[6][0][8], oracle[6][0][8], rel_tol=1e-10)


def test_full_size_weekly_contract_matches_the_oracle(native_executor) -> None:
    """The 52-node weekly contract at 2^20 + 2^20 paths (seed 11, domains 1 / 2)."""
    req = request(weekly(), paths=1 << 20)
    status, err, gpu = gpu_price(native_executor, req)
    assert status == 0, err.message
    assert_parity(gpu, _oracle.price_lsm_call(req, 32))


def test_fixtures_match_the_reference_values(native_executor) -> None:
    f = GOLDEN["insufficient_support_fixture"]
    t = f["schedule_times"]
    plan = dict(schedule_times=t, curve_times=t, log_discounts=f["log_discounts"], dividend_yield_times=t,
                cumulative_dividend_yields=[0.0] * 3, dividend_nodes=f["dividend_nodes"],
                dividend_amounts=f["dividend_amounts"], exercise_nodes=f["exercise_nodes"],
                expiry_node=f["expiry_node"], annualized_volatility=f["volatility"], dividend_policy=0)
    seeds = (tuple(f["training"]), tuple(f["evaluation"]))
    status, err, gpu = gpu_price(native_executor, request(plan, paths=4, seeds=seeds, support=1))
    assert status == 0, err.message
    assert gpu[5] == f["expected_exercise_counts"]
    assert gpu[6] == [(1, "insufficient_exercise_support", None, None, 3, None, 5, None, None, None, None)]
    status, err, _ = gpu_price(native_executor, request(plan, paths=4, seeds=seeds, support=0))
    assert status == _abi.FO_ERR_LSM
    assert err.message.decode() == ("continuation regression failed at exercise node 1: regression has 3 "
                                    "observations but degree 4 requires at least 5")
    o = GOLDEN["origin_decision_fixture"]
    plan.update(dividend_amounts=o["dividend_amounts"], exercise_nodes=o["exercise_nodes"],
                log_discounts=o["log_discounts"])
    status, err, gpu = gpu_price(native_executor, request(plan, S0=200.0, paths=1000, seeds=seeds))
    assert status == 0, err.message
    assert gpu[0] == o["expected_price"] and gpu[5] == o["expected_exercise_counts"]


def test_one_dividend_replications_reproduce_the_published_mean(native_executor) -> None:
    g = GOLDEN["one_dividend_statistical_pin"]
    steps = g["steps"]
    times = [n / steps for n in range(steps + 1)]
    plan = dict(schedule_times=times, curve_times=times,
                log_discounts=[0.0 if t == 0.0 else -g["rate"] * t for t in times], dividend_yield_times=times,
                cumulative_dividend_yields=[0.0] * (steps + 1), dividend_nodes=[steps // 2],
                dividend_amounts=[g["dividend"]], exercise_nodes=[steps // 2], expiry_node=steps,
                annualized_volatility=g["volatility"], dividend_policy=0)
    values = []
    for r in range(g["replications"]):
        seeds = ((g["training_seed_base"] + r, 1), (g["evaluation_seed_base"] + r, 2))
        status, err, gpu = gpu_price(native_executor, request(plan, paths=g["paths"], seeds=seeds))
        assert status == 0, err.message
        values.append(gpu[0])
    mean = sum(values) / len(values)
    assert abs(mean - g["published_mean"]) < 1e-8


def test_repeated_calls_are_bitwise_deterministic(native_executor) -> None:
    req = request(weekly(dividends=((13, 1.5),)), paths=50000)
    first = gpu_price(native_executor, req)[2]
    second = gpu_price(native_executor, req)[2]
    assert first == second


def test_overflowing_spot_reports_the_lowest_failing_path(native_executor) -> None:
    req = request(weekly(steps=4), S0=1.7e308, paths=64)
    status, err, _ = gpu_price(native_executor, req)
    with pytest.raises(_oracle.OracleFailure) as oracle_failure:
        _oracle.price_lsm_call(req, 1)
    assert status == _abi.FO_ERR_LSM
    assert err.code == _abi_code("FO_CODE_NON_FINITE_PATH_TRANSITION")
    assert err.path == oracle_failure.value.path
    node = oracle_failure.value.node
    assert err.message.decode().startswith(
        f"LSM training simulation failed: GBM path transition from node {node - 1} to {node} at path {err.path} "
        "produced non-finite spot from state ")


def _abi_code(name: str) -> int:
    import re

    text = (Path(__file__).resolve().parents[1] / "include" / "finoptions_cuda.h").read_text()
    block = text[text.index("typedef enum fo_error_code"): text.index("} fo_error_code;")]
    value = -1
    for m in re.finditer(r"(FO_CODE_\w+)(?:\s*=\s*(\d+))?", block):
        value = int(m.group(2)) if m.group(2) else value + 1
        if m.group(1) == name:
            return value
    raise KeyError(name)


def test_evaluation_outside_training_support_matches_the_oracle(native_executor) -> None:
    plan = weekly(steps=4, sigma=0.3, rate=0.0, q=0.0)
    for seed in range(200):
        req = request(plan, K=121.0, paths=8, seeds=((seed, 1), (seed + 1000, 2)))
        try:
            _oracle.price_lsm_call(req, 1)
            continue
        except _oracle.OracleFailure as failure:
            if failure.code != 21:  # evaluation outside training support
                continue
        status, err, _ = gpu_price(native_executor, req)
        assert status == _abi.FO_ERR_LSM
        assert err.code == _abi_code("FO_CODE_EVALUATION_OUTSIDE_TRAINING_SUPPORT")
        assert "active evaluation paths are in the money at node" in err.message.decode()
        return
    pytest.skip("no seed in range produced an unsupported evaluation row")
