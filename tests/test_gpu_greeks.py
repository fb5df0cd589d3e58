"""Pathwise adjoint Greeks (fo_price_lsm_call_greeks_f64 and the resident-plan form) on the B200.

The contract is the 52-week call of the weekly workload with two cash dividends of 1.5 at weeks 13
and 39 (liquidator), a continuous yield curve and r = 4%. The adjoint holds the fitted policy fixed,
so the exact check is a central finite difference of the fixed-policy price, obtained by
re-valuing the fitted plan on bumped markets (fo_lsm_call_plan_revalue_f64) with common random
numbers; the bump shrinks until no evaluation path changes its stopping row between the two sides.
The reference's own method, bump-and-reprice with a refit, is compared within its sampling error.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
from finoptions import _abi
from finoptions._requests import lsm_call_greeks, lsm_call_request, lsm_call_result

pytestmark = pytest.mark.gpu

NODES = 52
DIVIDEND_NODES = (13, 39)


def contract(paths: int, s0: float = 100.0, sigma: float = 0.25, log_discounts=None, dividends=(1.5, 1.5)) -> dict:
    t = [i / NODES for i in range(NODES + 1)]
    if log_discounts is None:
        log_discounts = [0.0 if i == 0 else -0.04 * t[i] for i in range(NODES + 1)]
    return dict(initial_spot=s0, strike=100.0, schedule_times=t, curve_times=t, log_discounts=list(log_discounts),
                dividend_yield_times=t, cumulative_dividend_yields=[0.0 if i == 0 else 0.02 * t[i] for i in range(NODES + 1)],
                dividend_nodes=list(DIVIDEND_NODES), dividend_amounts=list(dividends),
                exercise_nodes=list(range(NODES)), expiry_node=NODES, annualized_volatility=sigma, dividend_policy=0,
                training_paths=paths, evaluation_paths=paths, training_seed=11, training_domain=1, evaluation_seed=11,
                evaluation_domain=2, polynomial_degree=4, rank_tolerance=1e-12, condition_limit=1e8, tie_rule=0,
                insufficient_exercise_support=0)


def plain_price(native_executor, kwargs: dict) -> tuple:
    req = lsm_call_request(**kwargs)
    res = lsm_call_result(req.exercise_rows)
    err = _abi.FoError()
    assert _abi.load().fo_price_lsm_call_f64(native_executor.raw, ctypes.byref(req.struct), ctypes.byref(res.struct),
                                             ctypes.byref(err)) == 0, err.message
    return res.as_tuple()


class FittedPlan:
    """A resident plan with the Greeks enabled, fitted once on the base market."""

    def __init__(self, native_executor, kwargs: dict) -> None:
        self.lib = _abi.load()
        self.err = _abi.FoError()
        self.req = lsm_call_request(**kwargs)
        self.plan = ctypes.c_void_p()
        assert self.lib.fo_lsm_call_plan_create(native_executor.raw, ctypes.byref(self.req.struct),
                                                ctypes.byref(self.plan), ctypes.byref(self.err)) == 0, self.err.message
        assert self.lib.fo_lsm_call_plan_set_greeks(self.plan, 1, ctypes.byref(self.err)) == 0
        assert self.lib.fo_lsm_call_plan_launch(self.plan, ctypes.byref(self.err)) == 0, self.err.message
        res = lsm_call_result(self.req.exercise_rows)
        assert self.lib.fo_lsm_call_plan_collect(self.plan, ctypes.byref(res.struct), ctypes.byref(self.err)) == 0
        self.result = res.as_tuple()
        self.greeks = self.read_greeks()

    def read_greeks(self) -> tuple:
        g, d_l, d_d = lsm_call_greeks(NODES + 1, len(DIVIDEND_NODES))
        assert self.lib.fo_lsm_call_plan_greeks(self.plan, ctypes.byref(g), ctypes.byref(self.err)) == 0
        return g.delta, g.vega, d_l.copy(), d_d.copy()

    def revalue(self, kwargs: dict) -> tuple:
        req = lsm_call_request(**kwargs)
        res = lsm_call_result(req.exercise_rows)
        assert self.lib.fo_lsm_call_plan_revalue_f64(self.plan, ctypes.byref(req.struct), ctypes.byref(res.struct),
                                                     ctypes.byref(self.err)) == 0, self.err.message
        out = res.as_tuple()
        return out[0], tuple(out[5])

    def central_difference(self, bumped, h: float) -> float:
        for _ in range(8):
            (up, counts_up), (down, counts_down) = self.revalue(bumped(h)), self.revalue(bumped(-h))
            if counts_up == counts_down:
                return (up - down) / (2 * h)
            h /= 4
        pytest.fail("no bump small enough to keep every stopping row")
        return 0.0

    def close(self) -> None:
        self.lib.fo_lsm_call_plan_destroy(self.plan)


@pytest.fixture(scope="module")
def fitted(native_executor):
    plan = FittedPlan(native_executor, contract(1 << 18))
    yield plan
    plan.close()


@pytest.mark.parametrize("degree", [4, 2])
def test_greeks_pass_prices_exactly_like_the_plain_entry(native_executor, degree) -> None:
    kwargs = {**contract(1 << 16), "polynomial_degree": degree}
    req = lsm_call_request(**kwargs)
    res = lsm_call_result(req.exercise_rows)
    g, d_l, d_d = lsm_call_greeks(NODES + 1, 2)
    err = _abi.FoError()
    assert _abi.load().fo_price_lsm_call_greeks_f64(native_executor.raw, ctypes.byref(req.struct),
                                                    ctypes.byref(res.struct), ctypes.byref(g), ctypes.byref(err)) == 0
    got, want = res.as_tuple(), plain_price(native_executor, kwargs)
    assert got[:6] == want[:6]
    assert np.isfinite(d_l).all() and np.isfinite(d_d).all()


def _log_discount_bump(node: int):
    base = contract(1)["log_discounts"]
    return lambda e: [v + (e if i == node else 0.0) for i, v in enumerate(base)]


CASES = {
    "delta": (lambda e: dict(s0=100.0 + e), 1e-4),
    "vega": (lambda e: dict(sigma=0.25 + e), 2.5e-6),
    "dividend_13": (lambda e: dict(dividends=(1.5 + e, 1.5)), 1e-6),
    "dividend_39": (lambda e: dict(dividends=(1.5, 1.5 + e)), 1e-6),
    **{f"log_discount_{n}": ((lambda n: lambda e: dict(log_discounts=_log_discount_bump(n)(e)))(n), 1e-6)
       for n in (1, 12, 13, 14, 26, 39, 40, 51, 52)},
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_adjoint_matches_fixed_policy_central_differences(fitted, name: str) -> None:
    bump, h = CASES[name]
    delta, vega, d_l, d_d = fitted.greeks
    adjoint = {"delta": delta, "vega": vega, "dividend_13": d_d[0], "dividend_39": d_d[1],
               **{f"log_discount_{n}": d_l[n] for n in range(NODES + 1)}}[name]
    fd = fitted.central_difference(lambda e: contract(1 << 18, **bump(e)), h)
    # The finite difference carries the price's rounding over 2h and, at expiry, the payoff kink.
    assert abs(adjoint - fd) <= 2e-6 * abs(adjoint) + 2e-8, (adjoint, fd)


def test_log_discount_sensitivities_sum_to_the_price(fitted) -> None:
    """A parallel shift of the log-discount curve leaves every drift unchanged and scales every
    discount factor by exp(shift): its derivative is the price itself."""
    _, _, d_l, _ = fitted.greeks
    assert d_l.sum() == pytest.approx(fitted.result[0], rel=1e-12)


def test_revaluing_the_base_market_reproduces_the_price(fitted) -> None:
    price, counts = fitted.revalue(contract(1 << 18))
    assert price == fitted.result[0] and counts == tuple(fitted.result[5])


def test_refit_bump_and_reprice_agrees_within_its_sampling_error(native_executor, fitted) -> None:
    """The reference's method refits the policy at each bump. Refitted decisions add noise that
    grows as the bump shrinks, so it is compared at 1% (spot, volatility) and 0.2 (dividend) bumps,
    where it agrees with the fixed-policy adjoint within that noise."""
    delta, vega, _, d_d = fitted.greeks
    up = plain_price(native_executor, contract(1 << 18, s0=101.0))[0]
    down = plain_price(native_executor, contract(1 << 18, s0=99.0))[0]
    assert (up - down) / 2.0 == pytest.approx(delta, abs=0.03)
    up = plain_price(native_executor, contract(1 << 18, sigma=0.2525))[0]
    down = plain_price(native_executor, contract(1 << 18, sigma=0.2475))[0]
    assert (up - down) / 0.005 == pytest.approx(vega, rel=0.1)
    for j, bumped in enumerate(((1.7, 1.5), (1.5, 1.7))):
        lower = tuple(1.5 - (b - 1.5) for b in bumped)
        up = plain_price(native_executor, contract(1 << 18, dividends=bumped))[0]
        down = plain_price(native_executor, contract(1 << 18, dividends=lower))[0]
        assert (up - down) / 0.4 == pytest.approx(d_d[j], abs=0.05)


def test_torch_backward_returns_the_adjoint_greeks(executor, fitted) -> None:
    import finoptions as fo
    import torch

    base = contract(1 << 18)
    c = fo.LsmCallContract(
        strike=base["strike"], times=tuple(base["schedule_times"]), dividend_nodes=DIVIDEND_NODES,
        exercise_nodes=tuple(base["exercise_nodes"]), expiry_node=NODES,
        cumulative_yields=tuple(base["cumulative_dividend_yields"]), dividend_policy=fo.DividendPolicy.LIQUIDATOR,
        method=fo.Lsm(training_paths=1 << 18, evaluation_paths=1 << 18, training_stream=fo.RandomStream(seed=11, domain=1),
                      evaluation_stream=fo.RandomStream(seed=11, domain=2),
                      insufficient_exercise_support=fo.InsufficientExerciseSupportPolicy.FAIL),
        executor=executor)
    s0 = torch.tensor(100.0, dtype=torch.float64, requires_grad=True)
    sigma = torch.tensor(0.25, dtype=torch.float64, requires_grad=True)
    log_discounts = torch.tensor(base["log_discounts"], dtype=torch.float64, requires_grad=True)
    dividends = torch.tensor([1.5, 1.5], dtype=torch.float64, requires_grad=True)
    price = fo.lsm_call_price(s0, sigma, log_discounts, dividends, c)
    (2.0 * price).backward()
    delta, vega, d_l, d_d = fitted.greeks
    assert price.item() == fitted.result[0]
    assert s0.grad.item() == pytest.approx(2.0 * delta, rel=1e-14)
    assert sigma.grad.item() == pytest.approx(2.0 * vega, rel=1e-14)
    np.testing.assert_allclose(log_discounts.grad.numpy(), 2.0 * d_l, rtol=1e-14, atol=0)
    np.testing.assert_allclose(dividends.grad.numpy(), 2.0 * d_d, rtol=1e-14, atol=0)


def test_full_size_greeks_match_fixed_policy_differences(native_executor) -> None:
    """The contract at 2^20 + 2^20 paths: delta, vega and both dividend sensitivities."""
    plan = FittedPlan(native_executor, contract(1 << 20))
    try:
        delta, vega, _, d_d = plan.greeks
        for adjoint, bump, h in ((delta, lambda e: dict(s0=100.0 + e), 1e-4), (vega, lambda e: dict(sigma=0.25 + e), 2.5e-6),
                                 (d_d[0], lambda e: dict(dividends=(1.5 + e, 1.5)), 1e-6),
                                 (d_d[1], lambda e: dict(dividends=(1.5, 1.5 + e)), 1e-6)):
            fd = plan.central_difference(lambda e, b=bump: contract(1 << 20, **b(e)), h)
            assert abs(adjoint - fd) <= 2e-6 * abs(adjoint) + 2e-8, (adjoint, fd)
    finally:
        plan.close()
