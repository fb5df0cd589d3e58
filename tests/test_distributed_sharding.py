"""Grouped and ragged batches sharded over the ranks of a torch.distributed job (finoptions.distributed).

Two gloo ranks on the CPU stand in for two GPUs: each prices its block of groups (or contracts),
here through the oracle's restatement instead of the CUDA engine (no GPU), and the gathered result
must equal the oracle's unsharded result bit for bit, which holds because every group keeps its
random streams. A failure raised inside one shard must reach every rank with its row and group
moved to the whole batch; a request the single call rejects as a whole (overlapping stream domain
ranges) must be rejected on every rank; an exception outside the library on one rank must reach
every rank instead of leaving the others in the gather.
"""

from __future__ import annotations

import dataclasses
import datetime
import os
import socket

import _oracle
import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp
from _workloads import grouped_columns

import finoptions as fo
from finoptions.batch_lsm import _freeze
from finoptions.distributed import (
    group_block,
    grouped_weights,
    price_lsm_call_grouped_batch_sharded,
    price_lsm_call_ragged_sharded,
    shard_strike_groups,
    weighted_blocks,
)
from finoptions._requests import lsm_call_request, lsm_grouped_request
from _workloads import RaggedColumns, ragged_columns, ragged_row_as_call

PATHS = 2048
WORLD = 2


def public_request(states: int = 5):
    """A grouped batch over `states` states with 3 strikes each, explicit meshes, cash dividends."""
    c = grouped_columns(states, strikes_per_group=3, seed=31, min_exercise=4, max_exercise=10)
    groups = fo.LsmStrikeGroups(
        group_offsets=c.group_offsets, initial_spots=c.initial_spots, strikes=c.strikes, maturities=c.maturities,
        rates=c.rates, volatilities=c.volatilities,
        dividends=fo.CashDividendBatch(
            schedules=fo.RaggedCashDividends(offsets=c.dividend_offsets, times=c.dividend_times,
                                             amounts=c.dividend_amounts),
            policy=fo.DividendPolicy.LIQUIDATOR, maturity_boundary=fo.MaturityBoundary.STRICTLY_BEFORE))
    mesh = fo.ExplicitExerciseMesh(
        schedules=fo.RaggedExerciseTimes(offsets=c.exercise_offsets, times=c.exercise_times),
        origin_exercise=fo.OriginExercise.EXCLUDED)
    method = fo.Lsm(training_paths=PATHS, evaluation_paths=PATHS, training_stream=fo.RandomStream(seed=7, domain=100),
                    evaluation_stream=fo.RandomStream(seed=7, domain=900),
                    insufficient_exercise_support=fo.InsufficientExerciseSupportPolicy.CONTINUE)
    return groups, mesh, method


def oracle_pricer(*, groups, mesh, executor, method) -> fo.LsmBatchResult:
    """The same request priced by the oracle's restatement of the reference (CPU)."""
    d = groups.dividends
    request = lsm_grouped_request(
        group_offsets=groups.group_offsets, initial_spots=groups.initial_spots, strikes=groups.strikes,
        maturities=groups.maturities, rates=groups.rates, volatilities=groups.volatilities, dividend_model=1,
        dividend_offsets=d.schedules.offsets, dividend_times=d.schedules.times, dividend_amounts=d.schedules.amounts,
        dividend_policy=0, maturity_boundary=0, exercise_mesh=2, base_intervals=None, origin_exercise=0,
        explicit_exercise_offsets=mesh.schedules.offsets, explicit_exercise_times=mesh.schedules.times,
        training_paths=method.training_paths, evaluation_paths=method.evaluation_paths,
        training_seed=method.training_stream.seed, training_domain_start=method.training_stream.domain,
        evaluation_seed=method.evaluation_stream.seed, evaluation_domain_start=method.evaluation_stream.domain,
        polynomial_degree=method.polynomial_degree, rank_tolerance=method.rank_tolerance,
        condition_limit=method.condition_limit, tie_rule=0, insufficient_exercise_support=1)
    return _freeze(_oracle.price_lsm_grouped(request, 2))


FAILING_GROUP = 2


def failing_pricer(*, groups, mesh, executor, method) -> fo.LsmBatchResult:
    """Fails on the shard holding group FAILING_GROUP of the batch (domains 100 + group), at that
    group's second row."""
    lo = method.training_stream.domain - 100
    n = int(groups.initial_spots.size)
    if lo <= FAILING_GROUP < lo + n:
        local = FAILING_GROUP - lo
        exc = fo.LsmError(f"LSM batch estimator failed at row {int(groups.group_offsets[local]) + 1}: "
                          "regression rank deficient")
        exc.row, exc.group, exc.code = int(groups.group_offsets[local]) + 1, local, 321
        raise exc
    return oracle_pricer(groups=groups, mesh=mesh, executor=executor, method=method)


def broken_pricer(*, groups, mesh, executor, method) -> fo.LsmBatchResult:
    """Raises an exception outside the library's hierarchy on the shard that starts at group 0."""
    if method.training_stream.domain == 100:
        raise IndexError("offset table ended early")
    return oracle_pricer(groups=groups, mesh=mesh, executor=executor, method=method)


def ragged_public(contracts: int = 7):
    c = ragged_columns(contracts, seed=29, min_paths=256, max_paths=1024, min_exercise=4, max_exercise=9)
    return c, fo.LsmRaggedContracts(
        initial_spots=c.initial_spots, strikes=c.strikes, maturities=c.maturities, rates=c.rates,
        volatilities=c.volatilities, exercise=fo.RaggedExerciseTimes(offsets=c.exercise_offsets, times=c.exercise_times),
        training_paths=c.paths, evaluation_paths=c.paths.copy(), dividend_yields=c.dividend_yields,
        cash_dividends=fo.RaggedCashDividends(offsets=c.dividend_offsets, times=c.dividend_times,
                                              amounts=c.dividend_amounts))


RAGGED_METHOD = dict(insufficient_exercise_support=fo.InsufficientExerciseSupportPolicy.CONTINUE)


def oracle_ragged_pricer(*, contracts, origin_exercise, executor, training_stream, evaluation_stream,
                         **method) -> fo.LsmBatchResult:
    """Each contract priced alone by the oracle (domains start + row): prices, SD, SE and the
    stopping partition; the other columns stay zero."""
    cash = contracts.cash_dividends
    c = RaggedColumns(
        initial_spots=contracts.initial_spots, strikes=contracts.strikes, maturities=contracts.maturities,
        rates=contracts.rates, volatilities=contracts.volatilities, dividend_yields=contracts.dividend_yields,
        dividend_offsets=cash.offsets, dividend_times=cash.times, dividend_amounts=cash.amounts,
        exercise_offsets=contracts.exercise.offsets, exercise_times=contracts.exercise.times,
        paths=contracts.training_paths)
    columns = {name: np.zeros(c.rows, dtype=dtype) for name, dtype in RESULT_DTYPES.items()}
    for r in range(c.rows):
        kw = ragged_row_as_call(c, r, seed=training_stream.seed, support=1, training_domain=training_stream.domain,
                                evaluation_domain=evaluation_stream.domain)
        price, _, sd, se, _, counts, _ = _oracle.price_lsm_call(lsm_call_request(**kw), 1)
        columns["prices"][r], columns["sample_standard_deviations"][r], columns["standard_errors"][r] = price, sd, se
        columns["early_exercise_paths"][r], columns["expiry_paths"][r] = sum(counts[:-1]), counts[-1]
    for values in columns.values():
        values.flags.writeable = False
    return fo.LsmBatchResult(**columns)


RESULT_DTYPES = {"prices": np.float64, "sample_standard_deviations": np.float64, "standard_errors": np.float64,
                 "origin_decisions_fitted": np.bool_, "origin_exercised": np.bool_, "regression_nodes": np.uint32,
                 "no_training_support_nodes": np.uint32, "insufficient_exercise_support_nodes": np.uint32,
                 "minimum_in_the_money_training_paths": np.uint32,
                 "maximum_regression_condition_numbers": np.float64, "early_exercise_paths": np.uint32,
                 "expiry_paths": np.uint32}


def _attempt(fn, **kwargs):
    """(exception type name, message, row, group, code) of what fn raised, or None."""
    try:
        fn(**kwargs)
    except Exception as exc:  # noqa: BLE001 - the test inspects whatever reached this rank
        return (type(exc).__name__, str(exc), getattr(exc, "row", None), getattr(exc, "group", None),
                getattr(exc, "code", None))
    return None


def _worker(rank: int, port: int, queue) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        groups, mesh, method = public_request()
        result = price_lsm_call_grouped_batch_sharded(groups=groups, mesh=mesh, executor=None, method=method,
                                                      pricer=oracle_pricer)
        failure = _attempt(price_lsm_call_grouped_batch_sharded, groups=groups, mesh=mesh, executor=None,
                           method=method, pricer=failing_pricer)
        overlapping = dataclasses.replace(method, evaluation_stream=fo.RandomStream(seed=7, domain=103))
        rejected = _attempt(price_lsm_call_grouped_batch_sharded, groups=groups, mesh=mesh, executor=None,
                            method=overlapping, pricer=oracle_pricer)
        broken = _attempt(price_lsm_call_grouped_batch_sharded, groups=groups, mesh=mesh, executor=None,
                          method=method, pricer=broken_pricer)
        _, contracts = ragged_public()
        ragged = price_lsm_call_ragged_sharded(
            contracts=contracts, origin_exercise=fo.OriginExercise.EXCLUDED, executor=None,
            training_stream=fo.RandomStream(seed=41, domain=0), evaluation_stream=fo.RandomStream(seed=41, domain=5000),
            pricer=oracle_ragged_pricer, **RAGGED_METHOD)
        queue.put((rank, {name: np.asarray(getattr(result, name)) for name in ("prices", "standard_errors",
                                                                               "early_exercise_paths",
                                                                               "expiry_paths", "regression_nodes")},
                   failure, rejected, broken, np.asarray(ragged.prices), np.asarray(ragged.early_exercise_paths)))
    finally:
        dist.destroy_process_group()


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_group_blocks_cover_every_group_once() -> None:
    for groups in (0, 1, 5, 7, 4096):
        for world in (1, 2, 3, 8):
            blocks = [group_block(groups, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == groups
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:], strict=False))
            sizes = [hi - lo for lo, hi in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(fo.InputError):
        group_block(4, 2, 2)


def test_a_shard_prices_its_groups_like_the_whole_batch() -> None:
    groups, mesh, method = public_request()
    whole = oracle_pricer(groups=groups, mesh=mesh, executor=None, method=method)
    block, block_mesh, block_method = shard_strike_groups(groups, mesh, method, 2, 5)
    part = oracle_pricer(groups=block, mesh=block_mesh, executor=None, method=block_method)
    rows = slice(int(groups.group_offsets[2]), int(groups.group_offsets[5]))
    np.testing.assert_array_equal(part.prices, whole.prices[rows])
    np.testing.assert_array_equal(part.early_exercise_paths, whole.early_exercise_paths[rows])
    assert block_method.training_stream.domain == 102 and block_method.evaluation_stream.domain == 902


def test_weighted_blocks_cover_every_item_once_and_balance_the_work() -> None:
    rng = np.random.Generator(np.random.PCG64(3))
    for n in (0, 1, 5, 64, 1000):
        weights = rng.uniform(1.0, 100.0, n)
        for world in (1, 2, 3, 8):
            blocks = weighted_blocks(weights, world)
            assert len(blocks) == world and blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a[1] == b[0] and a[0] <= a[1] for a, b in zip(blocks, blocks[1:], strict=False))
            if n:
                loads = [weights[lo:hi].sum() for lo, hi in blocks]
                assert max(loads) <= weights.sum() / world + weights.max() + 1e-9
    groups, mesh, method = public_request()
    w = grouped_weights(groups, mesh, method)
    assert w.shape == (5,) and (w > 0).all()


def test_two_gloo_ranks_reproduce_the_single_call() -> None:
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, queue)) for r in range(WORLD)]
    for p in procs:
        p.start()
    outputs = [queue.get(timeout=240) for _ in range(WORLD)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    groups, mesh, method = public_request()
    whole = oracle_pricer(groups=groups, mesh=mesh, executor=None, method=method)
    _, contracts = ragged_public()
    ragged_whole = oracle_ragged_pricer(contracts=contracts, origin_exercise=fo.OriginExercise.EXCLUDED, executor=None,
                                        training_stream=fo.RandomStream(seed=41, domain=0),
                                        evaluation_stream=fo.RandomStream(seed=41, domain=5000), **RAGGED_METHOD)
    first_failing_row = int(groups.group_offsets[FAILING_GROUP]) + 1
    for _, columns, failure, rejected, broken, ragged_prices, ragged_early in outputs:
        for name, values in columns.items():
            np.testing.assert_array_equal(values, getattr(whole, name), err_msg=name)
        kind, message, row, group, code = failure
        assert (kind, row, group, code) == ("LsmError", first_failing_row, FAILING_GROUP, 321)
        assert f"at row {first_failing_row}:" in message
        # The whole request is validated on every rank: domains [100, 105) and [103, 108) overlap,
        # which neither shard's shifted, shorter ranges would show.
        assert rejected[0] == "InputError" and "overlap" in rejected[1], rejected
        assert broken[0] == "ExecutionError" and "IndexError: offset table ended early" in broken[1], broken
        np.testing.assert_array_equal(ragged_prices, ragged_whole.prices)
        np.testing.assert_array_equal(ragged_early, ragged_whole.early_exercise_paths)
