"""Grouped LSM batches spread over the GPUs of a torch.distributed job (one process per GPU).

The market states (groups) of a grouped batch are independent: group g simulates its own
training and evaluation populations on domains ``stream.domain + g``, and its strikes fit and
evaluate their policies on those populations alone. A batch therefore shards by group with no
collective on the data path. Rank r prices a contiguous block of groups with both stream domains
moved to the block's first group, so every group keeps its populations, and the row-ordered
result columns of the blocks are gathered in rank order (the only collective, on the results).
The gathered result equals the single-GPU call row for row, bit for bit.

When a shard fails, every rank raises the failure of the lowest failing shard, with its row and
group indices (``exc.row``, ``exc.group`` and the row named in the message) moved to the whole
batch. A single call would report the same failure whenever it is the batch's first one; when
several groups fail in different ways, a single call validates the whole request before pricing
and may name another one.
"""

from __future__ import annotations

import dataclasses
import re
from collections.abc import Callable

import numpy as np

from ._errors import BatchError, ExecutionError, InputError, LsmError, SimulationError
from .batch_lsm import (
    ContinuousDividendYieldBatch,
    ExerciseMesh,
    ExplicitExerciseMesh,
    LsmBatchResult,
    LsmStrikeGroups,
    RaggedExerciseTimes,
    price_lsm_call_grouped_batch,
)
from .dividends import RaggedCashDividends
from .lsm import Lsm
from .simulation import RandomStream

_RESULT_COLUMNS = tuple(f.name for f in dataclasses.fields(LsmBatchResult))
_ERRORS = {cls.__name__: cls for cls in (InputError, BatchError, LsmError, SimulationError, ExecutionError)}

type GroupedPricer = Callable[..., LsmBatchResult]


def group_block(groups: int, rank: int, world: int) -> tuple[int, int]:
    """The contiguous block [lo, hi) of groups that `rank` of `world` prices (sizes differ by at
    most one; a rank may get none when there are fewer groups than ranks)."""
    if world < 1 or not 0 <= rank < world or groups < 0:
        msg = f"rank {rank} of world {world} over {groups} groups is not a valid shard"
        raise InputError(msg)
    return groups * rank // world, groups * (rank + 1) // world


def _ragged_slice(offsets: np.ndarray, lo: int, hi: int) -> tuple[np.ndarray, int, int]:
    first, last = int(offsets[lo]), int(offsets[hi])
    return np.ascontiguousarray(offsets[lo:hi + 1] - first), first, last


def shard_strike_groups(groups: LsmStrikeGroups, mesh: ExerciseMesh, method: Lsm, lo: int,
                        hi: int) -> tuple[LsmStrikeGroups, ExerciseMesh, Lsm]:
    """The request that prices groups [lo, hi) of a grouped batch exactly as the whole batch
    prices them: per-group columns and ragged schedules sliced, strike rows of those groups, and
    both stream domains moved by `lo`."""
    count = int(groups.initial_spots.size)
    if not 0 <= lo < hi <= count:
        msg = f"group block [{lo}, {hi}) is outside the batch's {count} groups"
        raise InputError(msg)
    offsets = groups.group_offsets
    row_lo, row_hi = int(offsets[lo]), int(offsets[hi])
    d = groups.dividends
    if type(d) is ContinuousDividendYieldBatch:
        dividends = ContinuousDividendYieldBatch(annualized_decimals=np.ascontiguousarray(d.annualized_decimals[lo:hi]))
    else:
        sub, first, last = _ragged_slice(d.schedules.offsets, lo, hi)
        schedules = RaggedCashDividends(offsets=sub, times=np.ascontiguousarray(d.schedules.times[first:last]),
                                        amounts=np.ascontiguousarray(d.schedules.amounts[first:last]))
        dividends = dataclasses.replace(d, schedules=schedules)
    block = LsmStrikeGroups(
        group_offsets=np.ascontiguousarray((offsets[lo:hi + 1] - row_lo).astype(np.uint32)),
        initial_spots=np.ascontiguousarray(groups.initial_spots[lo:hi]),
        strikes=np.ascontiguousarray(groups.strikes[row_lo:row_hi]),
        maturities=np.ascontiguousarray(groups.maturities[lo:hi]),
        rates=np.ascontiguousarray(groups.rates[lo:hi]),
        volatilities=np.ascontiguousarray(groups.volatilities[lo:hi]),
        dividends=dividends,
    )
    if type(mesh) is ExplicitExerciseMesh:
        sub, first, last = _ragged_slice(mesh.schedules.offsets, lo, hi)
        mesh = ExplicitExerciseMesh(
            schedules=RaggedExerciseTimes(offsets=sub, times=np.ascontiguousarray(mesh.schedules.times[first:last])),
            origin_exercise=mesh.origin_exercise)
    method = dataclasses.replace(
        method,
        training_stream=RandomStream(seed=method.training_stream.seed, domain=method.training_stream.domain + lo),
        evaluation_stream=RandomStream(seed=method.evaluation_stream.seed,
                                       domain=method.evaluation_stream.domain + lo),
    )
    return block, mesh, method


def concatenate_results(parts: list[LsmBatchResult]) -> LsmBatchResult:
    """One immutable result whose rows are those of `parts` in order."""
    columns = {}
    for name in _RESULT_COLUMNS:
        values = np.concatenate([getattr(p, name) for p in parts])
        values.flags.writeable = False
        columns[name] = values
    return LsmBatchResult(**columns)


def _rebased(exc: Exception, row_offset: int, group_offset: int) -> tuple:
    row = int(getattr(exc, "row", -1))
    group = int(getattr(exc, "group", -1))
    message = str(exc)
    if row >= 0 and row_offset:
        message = re.sub(rf"\brow {row}\b", f"row {row + row_offset}", message, count=1)
    return (type(exc).__name__, message, row + row_offset if row >= 0 else -1,
            group + group_offset if group >= 0 else -1, int(getattr(exc, "code", 0)))


def price_lsm_call_grouped_batch_sharded(
    *,
    groups: LsmStrikeGroups,
    mesh: ExerciseMesh,
    executor: object,
    method: Lsm,
    process_group: object = None,
    pricer: GroupedPricer = price_lsm_call_grouped_batch,
) -> LsmBatchResult:
    """Price a grouped batch across the ranks of the default (or given) torch.distributed process
    group: every rank passes the whole request and its own executor (normally the CudaExecutor of
    its local GPU), prices its block of groups with `pricer`, and returns the whole result.

    Must be called by every rank of the group, like any collective. Works with the NCCL and gloo
    backends (results travel as Python objects).
    """
    import torch.distributed as dist  # noqa: PLC0415 - only distributed callers need torch

    if not dist.is_available() or not dist.is_initialized():
        msg = "price_lsm_call_grouped_batch_sharded needs an initialised torch.distributed process group"
        raise ExecutionError(msg)
    rank, world = dist.get_rank(process_group), dist.get_world_size(process_group)
    count = int(groups.initial_spots.size)
    lo, hi = group_block(count, rank, world)
    outcome: tuple
    try:
        if hi > lo:
            block, block_mesh, block_method = shard_strike_groups(groups, mesh, method, lo, hi)
            part = pricer(groups=block, mesh=block_mesh, executor=executor, method=block_method)
            outcome = ("ok", tuple(getattr(part, name) for name in _RESULT_COLUMNS))
        else:
            outcome = ("empty",)
    except (InputError, BatchError, LsmError, SimulationError, ExecutionError) as exc:
        outcome = ("error", *_rebased(exc, int(groups.group_offsets[lo]), lo))
    gathered: list = [None] * world
    dist.all_gather_object(gathered, outcome, group=process_group)
    for entry in gathered:
        if entry[0] == "error":
            _, kind, message, row, group, code = entry
            exc = _ERRORS[kind](message)
            exc.row, exc.group, exc.code = row, group, code  # type: ignore[attr-defined]
            raise exc
    parts = []
    for entry in gathered:
        if entry[0] == "ok":
            columns = {}
            for name, values in zip(_RESULT_COLUMNS, entry[1], strict=True):
                values = np.array(values, copy=True)  # a gathered copy arrives writeable
                values.flags.writeable = False
                columns[name] = values
            parts.append(LsmBatchResult(**columns))
    return concatenate_results(parts)


__all__ = ["concatenate_results", "group_block", "price_lsm_call_grouped_batch_sharded", "shard_strike_groups"]
