"""Central differences on the oracle with common random numbers, and their error bars.

The engine's adjoint differentiates every evaluation path's discounted payoff with the path's
stopping row held where the fitted policy put it. A central difference of a price over a bumped
market (S0 +- h, ...) agrees with that derivative path by path, except on "irregular" paths:

* paths whose stopping row on either side differs from the row the base market's policy chose
  (the policy, re-applied or refitted on the bumped market, moved the decision): their payoff
  jumps, or follows another branch than the one the adjoint differentiates;
* paths stopped at expiry whose payoff max(S_T - K, 0) is zero on exactly one side (the kink).

For a regular path the difference quotient fd_p equals the pathwise derivative up to O(h^2). So
|adjoint - FD| <= (sum over irregular paths of |fd_p| + |irregular| * G) / n, with G the largest
|fd_p| over the regular paths standing in for the irregular paths' unknown pathwise slopes. That
bound is each central difference's error bar. The regular paths alone give a tighter statement:
|adjoint - FD_regular| <= |irregular| * G / n, FD_regular = sum over regular paths of fd_p / n.
The jump term's statistical size, sqrt(sum over irregular paths of fd_p^2) / n, is reported beside
the hard bound: the jumps have either sign, so the difference is usually of that size.
A difference of two prices also carries their rounding: each is a running mean over n paths, good to
about sqrt(n) ulps of the price, which the 2h division magnifies.
"""

from __future__ import annotations

import os
from collections.abc import Callable
from dataclasses import dataclass

import _oracle
import numpy as np
from finoptions._requests import lsm_call_request

THREADS = max(1, min(32, os.cpu_count() or 1))

Bump = Callable[[dict, float], dict]


@dataclass(frozen=True)
class Difference:
    name: str
    h: float
    fd: float          # (P(+h) - P(-h)) / 2h
    bar: float         # error bar from the irregular paths
    irregular: int     # paths whose stopping row moved, or that cross the expiry kink
    moved: int         # of those, paths whose stopping row moved from the base market's
    fd_regular: float  # sum of the regular paths' difference quotients / n
    slope_bar: float   # |irregular| * G / n: bound on |adjoint - fd_regular|
    jump_sd: float     # sqrt(sum of the irregular paths' squared difference quotients) / n
    noise: float       # rounding of the two prices' running means, over 2h


def bumped(kwargs: dict, **changes) -> dict:
    return {**kwargs, **changes}


def spot_bump(kwargs: dict, e: float) -> dict:
    return bumped(kwargs, initial_spot=kwargs["initial_spot"] + e)


def vol_bump(kwargs: dict, e: float) -> dict:
    return bumped(kwargs, annualized_volatility=kwargs["annualized_volatility"] + e)


def log_discount_bump(node: int) -> Bump:
    def bump(kwargs: dict, e: float) -> dict:
        return bumped(kwargs, log_discounts=[v + (e if i == node else 0.0) for i, v in enumerate(kwargs["log_discounts"])])
    return bump


def dividend_bump(j: int) -> Bump:
    def bump(kwargs: dict, e: float) -> dict:
        return bumped(kwargs, dividend_amounts=[v + (e if i == j else 0.0) for i, v in enumerate(kwargs["dividend_amounts"])])
    return bump


def greek_cases(kwargs: dict, relative: float = 1e-4, absolute: float = 1e-6) -> list[tuple[str, float, Bump]]:
    """Delta and vega at a relative bump, every free log discount L_1.. L_N and every cash amount at an
    absolute bump (L_0 stays exactly 0)."""
    cases: list[tuple[str, float, Bump]] = [
        ("delta", relative * kwargs["initial_spot"], spot_bump),
        ("vega", relative * kwargs["annualized_volatility"], vol_bump),
    ]
    cases += [(f"L{i}", absolute, log_discount_bump(i)) for i in range(1, len(kwargs["schedule_times"]))]
    cases += [(f"D{j}", absolute, dividend_bump(j)) for j in range(len(kwargs["dividend_amounts"]))]
    return cases


def central_differences(kwargs: dict, cases: list[tuple[str, float, Bump]], *, mode: str,
                        base_stops: np.ndarray | None = None, threads: int = THREADS) -> dict[str, Difference]:
    """mode "frozen": every path stops at base_stops[p] on both sides; "fixed": the policy fitted on
    the base market is re-applied on each side; "refit": each side is priced from scratch. base_stops:
    every evaluation path's stopping row under the base market's fitted policy (computed here when
    not given)."""
    if base_stops is None:
        req = lsm_call_request(**kwargs)
        _, _, base = _oracle.price_markets(req, [req], refit=False, threads=threads)
        base_stops = base[0]
    base = lsm_call_request(**kwargs)
    markets = []
    for _, h, bump in cases:
        markets.append(lsm_call_request(**bump(kwargs, h)))
        markets.append(lsm_call_request(**bump(kwargs, -h)))
    prices, pay, stops = _oracle.price_markets(base, markets, refit=mode == "refit", threads=threads,
                                               frozen_stops=base_stops if mode == "frozen" else None)
    n = pay.shape[1]
    terminal = len(kwargs["exercise_nodes"])
    out = {}
    for i, (name, h, _) in enumerate(cases):
        up, down = 2 * i, 2 * i + 1
        fd_p = (pay[up] - pay[down]) / (2.0 * h)
        moved = (stops[up] != base_stops) | (stops[down] != base_stops)
        kink = (stops[up] == terminal) & (stops[down] == terminal) & ((pay[up] == 0.0) != (pay[down] == 0.0))
        irregular = moved | kink
        regular = ~irregular
        slope = float(np.abs(fd_p[regular]).max()) if regular.any() else 0.0
        slope_bar = int(irregular.sum()) * slope / n
        bar = float(np.abs(fd_p[irregular]).sum()) / n + slope_bar
        out[name] = Difference(name, h, (prices[up] - prices[down]) / (2.0 * h), bar, int(irregular.sum()),
                               int(moved.sum()), float(fd_p[regular].sum()) / n, slope_bar,
                               float(np.sqrt(np.square(fd_p[irregular]).sum())) / n,
                               4.0 * np.sqrt(n) * np.finfo(np.float64).eps * max(abs(prices[up]), abs(prices[down]))
                               / (2.0 * h))
    return out


def agrees(adjoint: float, d: Difference, rtol: float = 1e-6, atol: float = 2e-8) -> bool:
    """The price difference within its error bar and its rounding (each price is a running mean
    whose last bits, over 2h, grow with the price and the path count), and the regular paths' part
    - summed path by path, so free of that rounding - within its own bound."""
    tol = rtol * abs(adjoint) + atol
    return abs(adjoint - d.fd) <= d.bar + d.noise + tol and abs(adjoint - d.fd_regular) <= d.slope_bar + tol
