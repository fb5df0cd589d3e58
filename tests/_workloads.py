"""Seeded synthetic batch workloads shared by the batch tests and bench.py.

The grouped workload has the shapes of the reference's batched-LSM benchmark case: market states,
each with a uniform moneyness grid of strikes, exact explicit exercise meshes and exercise-aligned
cash dividends (crates/finoptions-lsm/src/batch/input.rs:594-723 for the column layout). Market
draws use NumPy's PCG64 with a fixed seed; the LSM paths themselves come from the engine's Philox
streams.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from finoptions._requests import GroupedRequest, lsm_grouped_request

TRAINING_DOMAIN_START = 0
EVALUATION_DOMAIN_START = 1 << 20
WEEKLY_INTERVALS = 52


def weekly_call_kwargs(paths: int = 1 << 20, *, dividends: bool = False) -> dict:
    """The weekly single-contract workload: S0 = K = 100, T = 1, grid t_i = i/52, exercise at nodes
    0..51 (the origin a common decision) plus expiry 52, log discounts -0.04 t, cumulative yield
    0.02 t, sigma = 0.25, Philox seed 11 with domains 1 / 2, degree 4, fail on insufficient support.
    dividends=True adds two cash dividends of 1.5 at weeks 13 and 39 (liquidator)."""
    n = WEEKLY_INTERVALS
    t = [i / n for i in range(n + 1)]
    return dict(
        initial_spot=100.0, strike=100.0, schedule_times=t, curve_times=t,
        log_discounts=[0.0 if i == 0 else -0.04 * t[i] for i in range(n + 1)], dividend_yield_times=t,
        cumulative_dividend_yields=[0.0 if i == 0 else 0.02 * t[i] for i in range(n + 1)],
        dividend_nodes=[13, 39] if dividends else [], dividend_amounts=[1.5, 1.5] if dividends else [],
        exercise_nodes=list(range(n)), expiry_node=n, annualized_volatility=0.25, dividend_policy=0,
        training_paths=paths, evaluation_paths=paths, training_seed=11, training_domain=1, evaluation_seed=11,
        evaluation_domain=2, polynomial_degree=4, rank_tolerance=1e-12, condition_limit=1e8, tie_rule=0,
        insufficient_exercise_support=0,
    )


@dataclass
class GroupedColumns:
    group_offsets: np.ndarray
    initial_spots: np.ndarray
    strikes: np.ndarray
    maturities: np.ndarray
    rates: np.ndarray
    volatilities: np.ndarray
    dividend_offsets: np.ndarray
    dividend_times: np.ndarray
    dividend_amounts: np.ndarray
    exercise_offsets: np.ndarray
    exercise_times: np.ndarray

    @property
    def groups(self) -> int:
        return int(self.initial_spots.size)

    @property
    def rows(self) -> int:
        return int(self.strikes.size)


def grouped_columns(groups: int, strikes_per_group: int = 8, seed: int = 23, min_exercise: int = 12,
                    max_exercise: int = 52, max_dividends: int = 4) -> GroupedColumns:
    """States S0~U[50,150], sigma~U[0.10,0.60], T~U[0.25,2.0], r~U[0,0.06], n~U{min..max}
    exercise dates at T*k/n (k = 1..n-1), 0..max_dividends cash dividends of U[0.5,3.0] at
    distinct exercise dates; strikes K = S0 * linspace(0.8, 1.2, strikes_per_group)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    s0 = rng.uniform(50.0, 150.0, groups)
    vol = rng.uniform(0.10, 0.60, groups)
    maturity = rng.uniform(0.25, 2.0, groups)
    rate = rng.uniform(0.0, 0.06, groups)
    n_ex = rng.integers(min_exercise, max_exercise + 1, groups)
    n_div = rng.integers(0, max_dividends + 1, groups)
    moneyness = np.linspace(0.8, 1.2, strikes_per_group)
    ex_offsets = [0]
    ex_times: list[float] = []
    div_offsets = [0]
    div_times: list[float] = []
    div_amounts: list[float] = []
    for g in range(groups):
        n = int(n_ex[g])
        times = [float(maturity[g]) * (k / n) for k in range(1, n)]
        ex_times.extend(times)
        ex_offsets.append(len(ex_times))
        k = min(int(n_div[g]), len(times))
        picks = np.sort(rng.choice(len(times), size=k, replace=False)) if k else np.array([], dtype=np.int64)
        div_times.extend(times[int(i)] for i in picks)
        div_amounts.extend(float(a) for a in rng.uniform(0.5, 3.0, k))
        div_offsets.append(len(div_times))
    return GroupedColumns(
        group_offsets=(np.arange(groups + 1, dtype=np.uint32) * strikes_per_group).astype(np.uint32),
        initial_spots=s0,
        strikes=(s0[:, None] * moneyness[None, :]).reshape(-1).copy(),
        maturities=maturity,
        rates=rate,
        volatilities=vol,
        dividend_offsets=np.asarray(div_offsets, dtype=np.int64),
        dividend_times=np.asarray(div_times, dtype=np.float64),
        dividend_amounts=np.asarray(div_amounts, dtype=np.float64),
        exercise_offsets=np.asarray(ex_offsets, dtype=np.int64),
        exercise_times=np.asarray(ex_times, dtype=np.float64),
    )


def grouped_request(c: GroupedColumns, paths: int, *, seed: int = 23, support: int = 1, degree: int = 4,
                    dividend_model: int = 1, grouped: bool = True, origin: int = 0,
                    volatility_convention: int = 0, maturity_boundary: int = 0) -> GroupedRequest:
    """Explicit-mesh request over the columns (cash dividends, liquidator, strictly-before maturity
    unless overridden). support 1 = continue (the reference benchmark's choice), 0 = fail."""
    cash = dividend_model != 0
    return lsm_grouped_request(
        group_offsets=c.group_offsets if grouped else None,
        initial_spots=c.initial_spots,
        strikes=c.strikes,
        maturities=c.maturities,
        rates=c.rates,
        volatilities=c.volatilities,
        dividend_model=dividend_model,
        dividend_yields=None if cash else np.zeros(c.groups),
        dividend_offsets=c.dividend_offsets if cash else None,
        dividend_times=c.dividend_times if cash else None,
        dividend_amounts=c.dividend_amounts if cash else None,
        dividend_policy=0,
        maturity_boundary=maturity_boundary,
        volatility_convention=volatility_convention,
        exercise_mesh=2,
        base_intervals=None,
        origin_exercise=origin,
        explicit_exercise_offsets=c.exercise_offsets,
        explicit_exercise_times=c.exercise_times,
        training_paths=paths,
        evaluation_paths=paths,
        training_seed=seed,
        training_domain_start=TRAINING_DOMAIN_START,
        evaluation_seed=seed,
        evaluation_domain_start=EVALUATION_DOMAIN_START,
        polynomial_degree=degree,
        rank_tolerance=1e-12,
        condition_limit=1e8,
        tie_rule=0,
        insufficient_exercise_support=support,
    )


def path_steps(c: GroupedColumns, paths: int) -> int:
    """Training + evaluation path-steps of a grouped request: paths x union-mesh intervals, both roles."""
    total = 0
    for g in range(c.groups):
        ex = c.exercise_times[c.exercise_offsets[g]:c.exercise_offsets[g + 1]]
        cash = c.dividend_times[c.dividend_offsets[g]:c.dividend_offsets[g + 1]]
        total += np.union1d(ex, cash).size + 1  # intervals: interior union times, then maturity
    return 2 * paths * total


@dataclass
class RaggedColumns:
    initial_spots: np.ndarray
    strikes: np.ndarray
    maturities: np.ndarray
    rates: np.ndarray
    volatilities: np.ndarray
    dividend_yields: np.ndarray
    dividend_offsets: np.ndarray
    dividend_times: np.ndarray
    dividend_amounts: np.ndarray
    exercise_offsets: np.ndarray
    exercise_times: np.ndarray
    paths: np.ndarray

    @property
    def rows(self) -> int:
        return int(self.initial_spots.size)


def ragged_columns(contracts: int, seed: int = 41, min_paths: int = 8192, max_paths: int = 262144,
                   min_exercise: int = 4, max_exercise: int = 104) -> RaggedColumns:
    """Independent contracts: P = floor(exp(U[ln min, ln max])) paths per role, n~U{min..max}
    exercise dates at T*k/n (k = 1..n-1), S0~U[20,500], K/S0~U[0.7,1.3], sigma~U[0.05,0.8],
    T~U[0.1,3], r~U[0,0.08]; even rows carry a continuous yield q~U[0,0.05], odd rows 1-6 cash
    dividends of U[0.1,5] at distinct exercise dates."""
    rng = np.random.Generator(np.random.PCG64(seed))
    paths = np.floor(np.exp(rng.uniform(np.log(min_paths), np.log(max_paths), contracts))).astype(np.uint64)
    n_ex = rng.integers(min_exercise, max_exercise + 1, contracts)
    s0 = rng.uniform(20.0, 500.0, contracts)
    moneyness = rng.uniform(0.7, 1.3, contracts)
    vol = rng.uniform(0.05, 0.8, contracts)
    maturity = rng.uniform(0.1, 3.0, contracts)
    rate = rng.uniform(0.0, 0.08, contracts)
    yields = np.where(np.arange(contracts) % 2 == 0, rng.uniform(0.0, 0.05, contracts), 0.0)
    ex_offsets, ex_times, div_offsets, div_times, div_amounts = [0], [], [0], [], []
    for r in range(contracts):
        n = int(n_ex[r])
        times = [float(maturity[r]) * (k / n) for k in range(1, n)]
        ex_times.extend(times)
        ex_offsets.append(len(ex_times))
        if r % 2 == 1 and times:
            k = min(int(rng.integers(1, 7)), len(times))
            picks = np.sort(rng.choice(len(times), size=k, replace=False))
            div_times.extend(times[int(i)] for i in picks)
            div_amounts.extend(float(a) for a in rng.uniform(0.1, 5.0, k))
        div_offsets.append(len(div_times))
    return RaggedColumns(
        initial_spots=s0, strikes=s0 * moneyness, maturities=maturity, rates=rate, volatilities=vol,
        dividend_yields=yields, dividend_offsets=np.asarray(div_offsets, dtype=np.int64),
        dividend_times=np.asarray(div_times, dtype=np.float64), dividend_amounts=np.asarray(div_amounts, dtype=np.float64),
        exercise_offsets=np.asarray(ex_offsets, dtype=np.int64), exercise_times=np.asarray(ex_times, dtype=np.float64),
        paths=paths)


def ragged_request(c: RaggedColumns, *, seed: int = 41, support: int = 1, training_domain_start: int = 0,
                   evaluation_domain_start: int = 1 << 20, degree: int = 4):
    from finoptions._requests import lsm_ragged_request

    return lsm_ragged_request(
        initial_spots=c.initial_spots, strikes=c.strikes, maturities=c.maturities, rates=c.rates,
        volatilities=c.volatilities, dividend_yields=c.dividend_yields, dividend_offsets=c.dividend_offsets,
        dividend_times=c.dividend_times, dividend_amounts=c.dividend_amounts, dividend_policy=0, maturity_boundary=0,
        exercise_offsets=c.exercise_offsets, exercise_times=c.exercise_times, origin_exercise=0,
        training_paths=c.paths, evaluation_paths=c.paths, training_seed=seed,
        training_domain_start=training_domain_start, evaluation_seed=seed,
        evaluation_domain_start=evaluation_domain_start, polynomial_degree=degree, rank_tolerance=1e-12,
        condition_limit=1e8, tie_rule=0, insufficient_exercise_support=support)


def explicit_call_kwargs(*, s0: float, strike: float, maturity: float, rate: float, dividend_yield: float,
                         volatility: float, exercise_times: np.ndarray, cash_times: np.ndarray,
                         cash_amounts: np.ndarray, paths: int, seed: int, training_domain: int,
                         evaluation_domain: int, support: int = 1, degree: int = 4) -> dict:
    """A contract of an explicit-mesh batch as single-contract arguments: the grid is the union of its
    exercise and cash times plus the origin and maturity, L = -r t, cumulative yield q t."""
    times = [0.0, *np.union1d(exercise_times, cash_times[cash_times < maturity]).tolist(), maturity]
    node = {t: i for i, t in enumerate(times)}
    return dict(
        initial_spot=s0, strike=strike, schedule_times=times, curve_times=times,
        log_discounts=[0.0 if i == 0 else -rate * t for i, t in enumerate(times)], dividend_yield_times=times,
        cumulative_dividend_yields=[0.0 if i == 0 else dividend_yield * t for i, t in enumerate(times)],
        dividend_nodes=[node[t] for t in cash_times.tolist()], dividend_amounts=cash_amounts.tolist(),
        exercise_nodes=[node[t] for t in exercise_times.tolist()], expiry_node=len(times) - 1,
        annualized_volatility=volatility, dividend_policy=0, training_paths=paths, evaluation_paths=paths,
        training_seed=seed, training_domain=training_domain, evaluation_seed=seed,
        evaluation_domain=evaluation_domain, polynomial_degree=degree, rank_tolerance=1e-12, condition_limit=1e8,
        tie_rule=0, insufficient_exercise_support=support)


def ragged_row_as_call(c: RaggedColumns, r: int, *, seed: int = 41, support: int = 1, training_domain: int = 0,
                       evaluation_domain: int = 1 << 20, degree: int = 4) -> dict:
    """Row r of a ragged batch as single-contract arguments (the union mesh of its exercise and cash
    times, domains start + r)."""
    cash = slice(c.dividend_offsets[r], c.dividend_offsets[r + 1])
    return explicit_call_kwargs(
        s0=float(c.initial_spots[r]), strike=float(c.strikes[r]), maturity=float(c.maturities[r]),
        rate=float(c.rates[r]), dividend_yield=float(c.dividend_yields[r]), volatility=float(c.volatilities[r]),
        exercise_times=c.exercise_times[c.exercise_offsets[r]:c.exercise_offsets[r + 1]],
        cash_times=c.dividend_times[cash], cash_amounts=c.dividend_amounts[cash], paths=int(c.paths[r]), seed=seed,
        training_domain=training_domain + r, evaluation_domain=evaluation_domain + r, support=support, degree=degree)


def grouped_row_as_call(c: GroupedColumns, row: int, paths: int, *, seed: int = 23, support: int = 1,
                        degree: int = 4) -> dict:
    """Strike row `row` of a grouped explicit-mesh workload as single-contract arguments: its state's
    mesh, market and populations (domains start + group)."""
    g = int(np.searchsorted(c.group_offsets, row, side="right")) - 1
    cash = slice(c.dividend_offsets[g], c.dividend_offsets[g + 1])
    return explicit_call_kwargs(
        s0=float(c.initial_spots[g]), strike=float(c.strikes[row]), maturity=float(c.maturities[g]),
        rate=float(c.rates[g]), dividend_yield=0.0, volatility=float(c.volatilities[g]),
        exercise_times=c.exercise_times[c.exercise_offsets[g]:c.exercise_offsets[g + 1]],
        cash_times=c.dividend_times[cash], cash_amounts=c.dividend_amounts[cash], paths=paths, seed=seed,
        training_domain=TRAINING_DOMAIN_START + g, evaluation_domain=EVALUATION_DOMAIN_START + g, support=support,
        degree=degree)


def ragged_path_steps(c: RaggedColumns) -> int:
    total = 0
    for r in range(c.rows):
        ex = c.exercise_times[c.exercise_offsets[r]:c.exercise_offsets[r + 1]]
        cash = c.dividend_times[c.dividend_offsets[r]:c.dividend_offsets[r + 1]]
        total += 2 * int(c.paths[r]) * (np.union1d(ex, cash).size + 1)
    return total
