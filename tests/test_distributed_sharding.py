"""Grouped batches sharded over the ranks of a torch.distributed job (finoptions.distributed).

Two gloo ranks on the CPU stand in for two GPUs: each prices its block of groups, here through
the oracle's grouped restatement instead of the CUDA engine (no GPU), and the gathered result must
equal the oracle's unsharded result bit for bit, which holds because every group keeps its random
streams. A failure raised inside one shard must reach every rank with its row and group moved to
the whole batch.
"""

from __future__ import annotations

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
from finoptions.distributed import group_block, price_lsm_call_grouped_batch_sharded, shard_strike_groups
from finoptions._requests import lsm_grouped_request

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


def failing_pricer(*, groups, mesh, executor, method) -> fo.LsmBatchResult:
    """Fails on the shard that starts at training domain 102 (groups 2.. of the batch), at its row 1."""
    if method.training_stream.domain == 102:
        exc = fo.LsmError("LSM batch estimator failed at row 1: regression rank deficient")
        exc.row, exc.group, exc.code = 1, 0, 321
        raise exc
    return oracle_pricer(groups=groups, mesh=mesh, executor=executor, method=method)


def _worker(rank: int, port: int, queue) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        groups, mesh, method = public_request()
        result = price_lsm_call_grouped_batch_sharded(groups=groups, mesh=mesh, executor=None, method=method,
                                                      pricer=oracle_pricer)
        try:
            price_lsm_call_grouped_batch_sharded(groups=groups, mesh=mesh, executor=None, method=method,
                                                 pricer=failing_pricer)
            failure = None
        except fo.LsmError as exc:
            failure = (str(exc), exc.row, exc.group, exc.code)
        queue.put((rank, {name: np.asarray(getattr(result, name)) for name in ("prices", "standard_errors",
                                                                               "early_exercise_paths",
                                                                               "expiry_paths", "regression_nodes")},
                   failure))
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
    first_failing_row = int(groups.group_offsets[2]) + 1
    for _, columns, failure in outputs:
        for name, values in columns.items():
            np.testing.assert_array_equal(values, getattr(whole, name), err_msg=name)
        message, row, group, code = failure
        assert (row, group, code) == (first_failing_row, 2, 321)
        assert f"at row {first_failing_row}:" in message
