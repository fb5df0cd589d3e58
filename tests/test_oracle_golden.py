"""Pin the CPU oracle against the reference's own known-answer vectors (tests/golden/golden.json).

Every value in golden.json was extracted from the reference's test sources by make_golden.py.
"""

from __future__ import annotations

import ctypes
import json
import math
from pathlib import Path

import numpy as np
import pytest
from finoptions._requests import lsm_call_request

import _oracle

GOLDEN = json.loads((Path(__file__).parent / "golden" / "golden.json").read_text())


def call_request(**overrides):
    base = dict(
        initial_spot=100.0, strike=100.0, schedule_times=[0.0, 0.5, 1.0], curve_times=[0.0, 0.5, 1.0],
        log_discounts=[0.0, -0.01, -0.025], dividend_yield_times=[0.0, 0.5, 1.0],
        cumulative_dividend_yields=[0.0, 0.0, 0.0], dividend_nodes=[1], dividend_amounts=[2.0], exercise_nodes=[1],
        expiry_node=2, annualized_volatility=0.2, dividend_policy=0, training_paths=4096, evaluation_paths=4096,
        training_seed=7, training_domain=1, evaluation_seed=7, evaluation_domain=2, polynomial_degree=4,
        rank_tolerance=1e-12, condition_limit=1e8, tie_rule=0, insufficient_exercise_support=0,
    )
    base.update(overrides)
    return lsm_call_request(**base)


def fixture_request(name: str, support: int):
    f = GOLDEN[name]
    t = f["schedule_times"]
    return call_request(
        initial_spot=f["initial_spot"], strike=f["strike"], schedule_times=t, curve_times=t,
        log_discounts=f["log_discounts"], dividend_yield_times=t, cumulative_dividend_yields=[0.0] * len(t),
        dividend_nodes=f["dividend_nodes"], dividend_amounts=f["dividend_amounts"], exercise_nodes=f["exercise_nodes"],
        expiry_node=f["expiry_node"], annualized_volatility=f["volatility"], training_paths=f["paths"],
        evaluation_paths=f["paths"], training_seed=f["training"][0], training_domain=f["training"][1],
        evaluation_seed=f["evaluation"][0], evaluation_domain=f["evaluation"][1], insufficient_exercise_support=support,
    )


def test_philox_matches_random123_known_answers() -> None:
    lib = _oracle.load()
    for case in GOLDEN["philox"]:
        counter = (ctypes.c_uint32 * 4)(*case["counter"])
        key = (ctypes.c_uint32 * 2)(*case["key"])
        out = (ctypes.c_uint32 * 4)()
        lib.orc_philox4x32_10(counter, key, out)
        assert list(out) == case["output"]


def test_zignor_reproduces_the_pinned_normal_bit_patterns() -> None:
    z = GOLDEN["zignor"]
    values = _oracle.normals(z["seed"], z["domain"], z["path"], 1, z["count"])[0]
    assert [int(b) for b in values.view(np.uint64)] == z["bits"]


def test_normal_budget_is_enforced() -> None:
    lib = _oracle.load()
    assert lib.orc_normal_after_budget(7, 11, 13, 1) == 1  # budget exhausted


def test_moment_kernels_match_exact_small_answers() -> None:
    lib = _oracle.load()
    m = GOLDEN["moments"]
    z, y, b = (np.array(m[k]) for k in ("predictors", "responses", "basis"))
    out = np.zeros(3)
    lib.orc_moments(z.ctypes.data, y.ctypes.data, b.ctypes.data, z.size, out.ctypes.data)
    assert list(out) == m["expected"]
    r = GOLDEN["recurrence_moments"]
    z, y, prev, cur = (np.array(r[k]) for k in ("predictors", "responses", "previous", "current"))
    nxt = np.zeros(2)
    lib.orc_recurrence_moments(z.ctypes.data, y.ctypes.data, prev.ctypes.data, cur.ctypes.data, nxt.ctypes.data,
                               z.size, r["alpha"], r["beta"], out.ctypes.data)
    assert list(nxt) == r["next"]
    assert list(out) == r["expected"]


def test_dividend_policies_have_the_reference_boundary_values() -> None:
    lib = _oracle.load()
    for policy, amount, before, after in GOLDEN["dividend_policy"]:
        code = 0 if policy == "liquidator" else 1
        assert lib.orc_apply_dividend(code, amount, before) == after


def test_exact_union_mesh_inserts_cash_times_without_rounding() -> None:
    lib = _oracle.load()
    case = GOLDEN["union_mesh"][0]
    cash = np.array(case["cash"])
    out = np.zeros(16)
    n = lib.orc_exact_union_times(case["maturity"], case["base_intervals"], cash.ctypes.data, cash.size,
                                  out.ctypes.data, out.size)
    assert list(out[:n]) == case["times"]
    below = np.array([np.nextafter(0.5, 0.0)])
    n = lib.orc_exact_union_times(1.0, 2, below.ctypes.data, 1, out.ctypes.data, out.size)
    assert list(out[:n]) == [0.0, below[0], 0.5, 1.0]


def test_declared_insufficient_support_fixture() -> None:
    f = GOLDEN["insufficient_support_fixture"]
    price, paths, _, _, nodes, counts, diags = _oracle.price_lsm_call(fixture_request("insufficient_support_fixture", 1), 1)
    assert paths == f["paths"]
    assert counts == f["expected_exercise_counts"]
    assert diags == [(1, "insufficient_exercise_support", None, None, f["expected_in_the_money_paths"], None,
                      f["expected_required_paths"], None, None, None, None)]
    with pytest.raises(_oracle.OracleFailure) as failure:
        _oracle.price_lsm_call(fixture_request("insufficient_support_fixture", 0), 1)
    assert failure.value.stage == 2  # fit
    assert failure.value.node == 1


def test_origin_exercise_is_one_common_decision() -> None:
    f = GOLDEN["origin_decision_fixture"]
    price, paths, sd, se, nodes, counts, diags = _oracle.price_lsm_call(fixture_request("origin_decision_fixture", 0), 2)
    assert price == f["expected_price"]
    assert counts == f["expected_exercise_counts"]
    assert (sd, se) == (0.0, 0.0)
    assert diags[0][1] == "origin_decision" and diags[0][2] is True


def test_one_dividend_replications_reproduce_the_published_summary() -> None:
    g = GOLDEN["one_dividend_statistical_pin"]
    steps = g["steps"]
    times = [n / steps for n in range(steps + 1)]
    log_discounts = [0.0 if t == 0.0 else -g["rate"] * t for t in times]
    values = []
    for replication in range(g["replications"]):
        q = call_request(
            schedule_times=times, curve_times=times, log_discounts=log_discounts, dividend_yield_times=times,
            cumulative_dividend_yields=[0.0] * (steps + 1), dividend_nodes=[steps // 2],
            dividend_amounts=[g["dividend"]], exercise_nodes=[steps // 2], expiry_node=steps,
            annualized_volatility=g["volatility"], training_paths=g["paths"], evaluation_paths=g["paths"],
            training_seed=g["training_seed_base"] + replication, training_domain=1,
            evaluation_seed=g["evaluation_seed_base"] + replication, evaluation_domain=2,
        )
        values.append(_oracle.price_lsm_call(q, 8)[0])
    count, mean, m2 = 0, 0.0, 0.0
    for v in values:
        count += 1
        delta = v - mean
        mean += delta / count
        m2 += delta * (v - mean)
    sd = math.sqrt(m2 / (count - 1))
    se = sd / math.sqrt(count)
    assert round(mean, 8) == g["published_mean"]
    assert round(sd, 8) == g["published_replication_sd"]
    assert round(se, 8) == g["published_standard_error"]
    half = g["student_t_99_df_11"] * se
    assert mean - half <= g["reference_value"] <= mean + half


def test_oracle_threads_do_not_change_results() -> None:
    q = call_request(training_paths=20000, evaluation_paths=20000)
    assert _oracle.price_lsm_call(q, 1) == _oracle.price_lsm_call(q, 8)


def test_continuous_yield_european_slice_covers_black_scholes_merton() -> None:
    spot, strike, rate, q_yield, sigma, maturity = 100.0, 105.0, 0.05, 0.02, 0.25, 1.25
    q = call_request(
        initial_spot=spot, strike=strike, schedule_times=[0.0, maturity], curve_times=[0.0, maturity],
        log_discounts=[0.0, -rate * maturity], dividend_yield_times=[0.0, maturity],
        cumulative_dividend_yields=[0.0, q_yield * maturity], dividend_nodes=[], dividend_amounts=[], exercise_nodes=[],
        expiry_node=1, annualized_volatility=sigma, training_paths=131072, evaluation_paths=131072,
        training_seed=10000, training_domain=1, evaluation_seed=20000, evaluation_domain=2,
    )
    price, _, _, se, _, _, diags = _oracle.price_lsm_call(q, 8)
    srt = sigma * math.sqrt(maturity)
    d1 = (math.log(spot / strike) + (rate - q_yield + 0.5 * sigma**2) * maturity) / srt
    cdf = lambda x: 0.5 * math.erfc(-x / math.sqrt(2.0))  # noqa: E731
    expected = spot * math.exp(-q_yield * maturity) * cdf(d1) - strike * math.exp(-rate * maturity) * cdf(d1 - srt)
    assert abs(price - expected) <= 5.0 * se
    assert diags == []


def _explicit_normals_request(paths: int, dividend: tuple[int, float] | None = None, exercises=(1, 2)):
    from finoptions._requests import gbm_seeded_request

    times = [0.0, 0.25, 0.5, 1.0]
    return gbm_seeded_request(
        initial_spot=100.0, schedule_times=times, curve_times=times, log_discounts=[0.0, -0.01, -0.02, -0.05],
        dividend_yield_times=times, cumulative_dividend_yields=[0.0] * 4,
        dividend_nodes=[] if dividend is None else [dividend[0]], dividend_amounts=[] if dividend is None else [dividend[1]],
        exercise_nodes=list(exercises), expiry_node=3, annualized_volatility=0.20, dividend_policy=0, paths=paths,
        seed=0, domain=0,
    )


def test_explicit_normal_paths_follow_the_adjacent_transition() -> None:
    """The reference's tests/test_simulation.py:59-96 closed form: S *= exp(-(dL) - v/2 + sqrt(v) z)."""
    normals = np.array([[0.0, 1.0], [0.5, -0.5], [-1.0, 0.25]])
    states = _oracle.simulate_from(_explicit_normals_request(2), normals)
    times, logs = (0.0, 0.25, 0.5, 1.0), (0.0, -0.01, -0.02, -0.05)
    current, want = np.full(2, 100.0), []
    for i in range(3):
        variance = 0.2**2 * (times[i + 1] - times[i])
        current = current * np.exp(-(logs[i + 1] - logs[i]) - 0.5 * variance + np.sqrt(variance) * normals[i])
        want.append(current.copy())
    np.testing.assert_allclose(states, np.array(want), rtol=2e-15, atol=0.0)


def test_explicit_normal_paths_store_the_pre_dividend_exercise_state() -> None:
    """tests/test_simulation.py:99-116: a same-node dividend is applied after the exercise observation."""
    states = _oracle.simulate_from(_explicit_normals_request(1, dividend=(1, 200.0), exercises=(1,)), np.zeros((3, 1)))
    assert states[0, 0] > 0.0 and states[1, 0] == 0.0


def test_explicit_normal_paths_reject_the_first_non_finite_variate() -> None:
    """tests/test_simulation.py:136-139: the first bad variate in [interval][path] order is reported."""
    normals = np.zeros((3, 2))
    normals[2, 1] = np.nan
    normals[2, 0] = np.inf
    with pytest.raises(_oracle.OracleFailure) as failure:
        _oracle.simulate_from(_explicit_normals_request(2), normals)
    assert failure.value.path == 0 and "interval=2" in str(failure.value)
