"""Adjoint Greeks against the oracle (the CPU restatement of the reference), at the stated bumps.

The contract is the 52-week call with two cash dividends of 1.5 at weeks 13 and 39 (liquidator),
r = 4% as log discounts, a 2% continuous-yield curve and sigma = 0.25. Every Greek the adjoint
returns is checked (delta, vega, dP/dL_i for the 52 free log discounts L_1..L_52, both dividend
sensitivities) at relative bumps of 1e-4 on S0 and sigma and absolute bumps of 1e-6 on each L_i
and D_j, with common random numbers, three ways (tests/_fd.py gives the error bars):

1. frozen: oracle central differences with every evaluation path's stopping row frozen at the row
   the fitted policy chose on the base market - the quantity the adjoint forms, so the two agree to
   rounding;
2. fixed policy: oracle central differences with the base market's fitted policy re-applied on each
   bumped market (FittedLsmCallPolicy::evaluate, policy.rs:642-834); paths whose stopping row the
   bump moves make the error bar;
3. refit: the reference's own method, bump-and-reprice with the policy refitted on both sides
   (two price_lsm_call calls on identical streams, policy.rs:306-336), with the same error bar.

The engine's own fixed-policy revaluation (fo_lsm_call_plan_revalue_f64) is also checked against
the oracle's on every bumped market, and the engine's per-path stopping rows against the oracle's.
"""

from __future__ import annotations

import ctypes

import _fd
import _oracle
import numpy as np
import pytest
from _workloads import ragged_columns, ragged_request, ragged_row_as_call, weekly_call_kwargs
from finoptions import _abi
from finoptions._requests import batch_columns, lsm_call_greeks, lsm_call_request, lsm_call_result

pytestmark = pytest.mark.gpu

NODES = 52
PATHS = 1 << 16


def contract(paths: int = PATHS) -> dict:
    return weekly_call_kwargs(paths, dividends=True)


class GpuPlan:
    """A resident plan with the adjoint enabled: fitted once on the base market."""

    def __init__(self, native_executor, kwargs: dict) -> None:
        self.lib = _abi.load()
        self.err = _abi.FoError()
        self.kwargs = kwargs
        self.req = lsm_call_request(**kwargs)
        self.plan = ctypes.c_void_p()
        assert self.lib.fo_lsm_call_plan_create(native_executor.raw, ctypes.byref(self.req.struct),
                                                ctypes.byref(self.plan), ctypes.byref(self.err)) == 0, self.err.message
        assert self.lib.fo_lsm_call_plan_set_greeks(self.plan, 1, ctypes.byref(self.err)) == 0
        assert self.lib.fo_lsm_call_plan_launch(self.plan, ctypes.byref(self.err)) == 0, self.err.message
        res = lsm_call_result(self.req.exercise_rows)
        assert self.lib.fo_lsm_call_plan_collect(self.plan, ctypes.byref(res.struct), ctypes.byref(self.err)) == 0
        self.result = res.as_tuple()
        g, d_l, d_d = lsm_call_greeks(len(kwargs["schedule_times"]), len(kwargs["dividend_amounts"]))
        assert self.lib.fo_lsm_call_plan_greeks(self.plan, ctypes.byref(g), ctypes.byref(self.err)) == 0
        self.greeks = {"delta": g.delta, "vega": g.vega,
                       **{f"L{i}": float(d_l[i]) for i in range(len(d_l))},
                       **{f"D{j}": float(d_d[j]) for j in range(len(kwargs["dividend_amounts"]))}}

    def stopping_rows(self) -> np.ndarray:
        rows = np.zeros(self.kwargs["evaluation_paths"], dtype=np.uint32)
        assert self.lib.fo_lsm_call_plan_stopping_rows(self.plan, rows.ctypes.data, rows.size,
                                                       ctypes.byref(self.err)) == 0, self.err.message
        return rows

    def revalue(self, kwargs: dict) -> float:
        req = lsm_call_request(**kwargs)
        res = lsm_call_result(req.exercise_rows)
        assert self.lib.fo_lsm_call_plan_revalue_f64(self.plan, ctypes.byref(req.struct), ctypes.byref(res.struct),
                                                     ctypes.byref(self.err)) == 0, self.err.message
        return res.as_tuple()[0]

    def close(self) -> None:
        self.lib.fo_lsm_call_plan_destroy(self.plan)


@pytest.fixture(scope="module")
def dividend_contract(native_executor):
    kwargs = contract()
    plan = GpuPlan(native_executor, kwargs)
    _, _, base_stops = _oracle.price_markets(lsm_call_request(**kwargs), [lsm_call_request(**kwargs)], refit=False)
    yield plan, base_stops[0]
    plan.close()


def _report(title: str, plan: GpuPlan, diffs: dict[str, _fd.Difference]) -> None:
    print(f"\n[greeks-oracle] {title}: name adjoint fd bar jump_sd fd_regular irregular moved")
    for name, d in diffs.items():
        print(f"[greeks-oracle]   {name} {plan.greeks[name]:.12g} {d.fd:.12g} {d.bar:.3g} {d.jump_sd:.3g} "
              f"{d.fd_regular:.12g} {d.irregular} {d.moved}")


def test_policy_and_stopping_rows_match_the_oracle(dividend_contract) -> None:
    """Same price and stopping counts as the oracle, and no path stops at a different row."""
    plan, oracle_stops = dividend_contract
    want = _oracle.price_lsm_call(plan.req, _fd.THREADS)
    assert plan.result[0] == pytest.approx(want[0], rel=1e-9)
    assert plan.result[3] == pytest.approx(want[3], rel=1e-9)
    assert plan.result[5] == want[5]
    assert int((plan.stopping_rows() != oracle_stops).sum()) == 0


def test_adjoint_matches_frozen_stop_differences_of_the_oracle(dividend_contract) -> None:
    plan, oracle_stops = dividend_contract
    cases = _fd.greek_cases(plan.kwargs)
    assert len(cases) == 2 + NODES + 2
    diffs = _fd.central_differences(plan.kwargs, cases, mode="frozen", base_stops=oracle_stops)
    _report("frozen stopping rows", plan, diffs)
    bad = [(n, plan.greeks[n], d) for n, d in diffs.items() if not _fd.agrees(plan.greeks[n], d)]
    assert not bad, bad
    # Frozen rows leave only expiry-kink paths irregular: under 0.1% of the paths.
    assert max(d.irregular for d in diffs.values()) <= PATHS // 1000


def test_adjoint_matches_fixed_policy_differences_within_their_error_bars(dividend_contract) -> None:
    plan, _ = dividend_contract
    cases = _fd.greek_cases(plan.kwargs)
    diffs = _fd.central_differences(plan.kwargs, cases, mode="fixed")
    _report("fixed policy", plan, diffs)
    bad = [(n, plan.greeks[n], d) for n, d in diffs.items() if not _fd.agrees(plan.greeks[n], d)]
    assert not bad, bad


def test_engine_revaluation_matches_the_oracle_on_every_bumped_market(dividend_contract) -> None:
    plan, _ = dividend_contract
    markets = []
    for _, h, bump in _fd.greek_cases(plan.kwargs):
        markets += [bump(plan.kwargs, h), bump(plan.kwargs, -h)]
    want, _, _ = _oracle.price_markets(lsm_call_request(**plan.kwargs), [lsm_call_request(**m) for m in markets],
                                       refit=False, paths=False, threads=_fd.THREADS)
    got = np.array([plan.revalue(m) for m in markets])
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=0)


def test_adjoint_matches_the_references_bump_and_reprice_within_its_error_bars(dividend_contract) -> None:
    plan, _ = dividend_contract
    cases = _fd.greek_cases(plan.kwargs)
    diffs = _fd.central_differences(plan.kwargs, cases, mode="refit")
    _report("refit bump-and-reprice", plan, diffs)
    bad = [(n, plan.greeks[n], d) for n, d in diffs.items() if not _fd.agrees(plan.greeks[n], d)]
    assert not bad, bad


# ---- ragged rows of the benchmark workload (1,024 contracts, seed 41) ---------------------------

def _ragged_greeks(native_executor, c):
    nodes = [len(ragged_row_as_call(c, r)["schedule_times"]) for r in range(c.rows)]
    g = _abi.FoRaggedGreeksColumns()
    delta, vega = np.zeros(c.rows), np.zeros(c.rows)
    d_l, offsets = np.zeros(sum(nodes)), np.zeros(c.rows + 1, dtype=np.int64)
    d_d = np.zeros(max(c.dividend_times.size, 1))
    dp = ctypes.POINTER(ctypes.c_double)
    g.delta, g.vega = delta.ctypes.data_as(dp), vega.ctypes.data_as(dp)
    g.log_discount_sensitivities = d_l.ctypes.data_as(dp)
    g.log_discount_capacity = d_l.size
    g.log_discount_offsets = offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    g.dividend_sensitivities = d_d.ctypes.data_as(dp)
    req = ragged_request(c)
    cols = batch_columns(req.rows)
    err = _abi.FoError()
    assert _abi.load().fo_price_lsm_ragged_f64(native_executor.raw, ctypes.byref(req.struct),
                                               ctypes.byref(cols.struct), ctypes.byref(g), ctypes.byref(err)) == 0, \
        err.message
    return cols.as_tuple(), delta, vega, d_l, offsets, d_d


def _sample_rows(c) -> list[int]:
    """A cash-dividend row and a continuous-yield row with the fewest paths, and the row with the
    most exercise dates among those up to 20,000 paths."""
    n_ex = np.diff(c.exercise_offsets)
    odd = [r for r in range(c.rows) if r % 2 == 1]
    even = [r for r in range(c.rows) if r % 2 == 0]
    small = [r for r in range(c.rows) if c.paths[r] <= 20000]
    return sorted({min(odd, key=lambda r: c.paths[r]), min(even, key=lambda r: c.paths[r]),
                   max(small, key=lambda r: n_ex[r])})


def test_benchmark_ragged_rows_greeks_match_the_oracle(native_executor) -> None:
    c = ragged_columns(1024, seed=41)
    _, delta, vega, d_l, offsets, d_d = _ragged_greeks(native_executor, c)
    for r in _sample_rows(c):
        kwargs = ragged_row_as_call(c, r)
        first = int(c.dividend_offsets[r])
        adjoint = {"delta": delta[r], "vega": vega[r],
                   **{f"L{i}": float(v) for i, v in enumerate(d_l[offsets[r]:offsets[r + 1]])},
                   **{f"D{j}": float(d_d[first + j]) for j in range(len(kwargs["dividend_amounts"]))}}
        cases = _fd.greek_cases(kwargs)
        _, _, stops = _oracle.price_markets(lsm_call_request(**kwargs), [lsm_call_request(**kwargs)], refit=False)
        for mode in ("frozen", "fixed", "refit"):
            diffs = _fd.central_differences(kwargs, cases, mode=mode, base_stops=stops[0])
            print(f"\n[greeks-oracle] ragged row {r} ({c.paths[r]} paths, {len(cases)} Greeks) {mode}: "
                  f"max irregular {max(d.irregular for d in diffs.values())}")
            bad = [(n, adjoint[n], d) for n, d in diffs.items() if not _fd.agrees(adjoint[n], d)]
            assert not bad, (r, mode, bad)
