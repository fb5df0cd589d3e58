"""Grouped and ragged LSM batches spread over the GPUs of a torch.distributed job (one process per GPU).

The market states (groups) of a grouped batch are independent: group g simulates its own
training and evaluation populations on domains ``stream.domain + g``, and its strikes fit and
evaluate their policies on those populations alone. The contracts of a ragged batch are
independent the same way (row r on domains ``stream.domain + r``). A batch therefore shards with
no collective on the data path. Rank r prices a contiguous block of groups (rows) with both
stream domains moved to the block's first group, so every group keeps its populations, and the
row-ordered result columns of the blocks are gathered in rank order (the only collective, on the
results). The gathered result equals the single-GPU call row for row, bit for bit.

Blocks are balanced on the work they carry, sum over the block's problems of (training +
evaluation paths) x grid intervals, not on their group counts: the block boundaries sit at the
quantiles of that prefix sum, so no rank's block exceeds an equal share by more than one group's
work. (A longest-processing-time assignment would give ranks non-contiguous groups, whose domains
``start + g`` one call with a single domain start cannot address.)

Every rank first validates the whole request (validate_lsm_call_grouped_batch /
validate_lsm_call_ragged), so a request the single call rejects - e.g. training and evaluation
domain ranges that overlap over all groups, which no shard sees alone - is rejected identically on
every rank. When a shard fails, every rank raises the failure of the lowest failing shard, with its
row and group indices (``exc.row``, ``exc.group`` and the row named in the message) moved to the
whole batch; any other exception on a rank reaches every rank as an ExecutionError naming it, so no
rank is left waiting in the gather.
"""

from __future__ import annotations

import dataclasses
import re
from collections.abc import Callable

import numpy as np

from ._errors import BatchError, ExecutionError, InputError, LsmError, SimulationError
from .batch_lsm import (
    CashDividendExerciseMesh,
    ContinuousDividendYieldBatch,
    ExerciseMesh,
    ExplicitExerciseMesh,
    LsmBatchResult,
    LsmRaggedContracts,
    LsmRaggedGreeks,
    LsmStrikeGroups,
    OriginExercise,
    RaggedExerciseTimes,
    UniformExerciseMesh,
    price_lsm_call_grouped_batch,
    price_lsm_call_ragged,
    price_lsm_call_ragged_greeks,
    validate_lsm_call_grouped_batch,
    validate_lsm_call_ragged,
)
from .dividends import RaggedCashDividends
from .lsm import Lsm
from .simulation import RandomStream

_RESULT_COLUMNS = tuple(f.name for f in dataclasses.fields(LsmBatchResult))
_LIBRARY_ERRORS = (InputError, BatchError, LsmError, SimulationError, ExecutionError)
_ERRORS = {cls.__name__: cls for cls in _LIBRARY_ERRORS}

type GroupedPricer = Callable[..., LsmBatchResult]


def group_block(groups: int, rank: int, world: int) -> tuple[int, int]:
    """The contiguous block [lo, hi) of an equal-count split (sizes differ by at most one; a rank
    may get none when there are fewer groups than ranks)."""
    if world < 1 or not 0 <= rank < world or groups < 0:
        msg = f"rank {rank} of world {world} over {groups} groups is not a valid shard"
        raise InputError(msg)
    return groups * rank // world, groups * (rank + 1) // world


def weighted_blocks(weights: np.ndarray, world: int) -> list[tuple[int, int]]:
    """Contiguous blocks [lo, hi) covering every item once, one per rank, whose boundaries sit at
    the world-quantiles of the weights' prefix sum (each at the nearer of the two items around the
    quantile): a block's weight exceeds total / world by at most one item's weight."""
    if world < 1:
        msg = f"world {world} is not a valid shard count"
        raise InputError(msg)
    w = np.asarray(weights, dtype=np.float64)
    n = int(w.size)
    prefix = np.concatenate([[0.0], np.cumsum(w)])
    total = float(prefix[-1])
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        i = int(np.searchsorted(prefix, target, side="left"))
        if i > 0 and target - prefix[i - 1] < prefix[min(i, n)] - target:
            i -= 1
        bounds.append(min(max(i, bounds[-1]), n))
    bounds.append(n)
    return list(zip(bounds[:-1], bounds[1:], strict=True))


def _intervals(exercise_counts: np.ndarray, cash_counts: np.ndarray, mesh: ExerciseMesh) -> np.ndarray:
    """Grid intervals of each group's mesh (an upper bound where exercise and cash times merge)."""
    if type(mesh) is UniformExerciseMesh:
        return mesh.base_intervals + cash_counts
    if type(mesh) is CashDividendExerciseMesh:
        return cash_counts + 1
    return exercise_counts + cash_counts + 1


def grouped_weights(groups: LsmStrikeGroups, mesh: ExerciseMesh, method: Lsm) -> np.ndarray:
    """Per group: (training + evaluation paths) x grid intervals x strikes."""
    count = int(groups.initial_spots.size)
    strikes = np.diff(groups.group_offsets.astype(np.int64))
    d = groups.dividends
    cash = (np.zeros(count, dtype=np.int64) if type(d) is ContinuousDividendYieldBatch
            else np.diff(d.schedules.offsets.astype(np.int64)))
    exercise = (np.diff(mesh.schedules.offsets.astype(np.int64)) if type(mesh) is ExplicitExerciseMesh
                else np.zeros(count, dtype=np.int64))
    paths = method.training_paths + method.evaluation_paths
    return paths * _intervals(exercise, cash, mesh).astype(np.float64) * strikes


def ragged_weights(contracts: LsmRaggedContracts) -> np.ndarray:
    """Per contract: (training + evaluation paths) x grid intervals."""
    exercise = np.diff(contracts.exercise.offsets.astype(np.int64))
    cash = contracts.cash_dividends
    cash_counts = np.zeros(contracts.rows, dtype=np.int64) if cash is None else np.diff(cash.offsets.astype(np.int64))
    paths = contracts.training_paths.astype(np.float64) + contracts.evaluation_paths.astype(np.float64)
    return paths * (exercise + cash_counts + 1)


def _ragged_slice(offsets: np.ndarray, lo: int, hi: int) -> tuple[np.ndarray, int, int]:
    first, last = int(offsets[lo]), int(offsets[hi])
    return np.ascontiguousarray(offsets[lo:hi + 1] - first), first, last


def _shifted(stream: RandomStream, by: int) -> RandomStream:
    return RandomStream(seed=stream.seed, domain=stream.domain + by)


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
    method = dataclasses.replace(method, training_stream=_shifted(method.training_stream, lo),
                                 evaluation_stream=_shifted(method.evaluation_stream, lo))
    return block, mesh, method


def shard_ragged_contracts(contracts: LsmRaggedContracts, lo: int, hi: int) -> LsmRaggedContracts:
    """Contracts [lo, hi) of a ragged batch with their ragged schedules sliced (the caller moves
    both stream domains by `lo`)."""
    if not 0 <= lo < hi <= contracts.rows:
        msg = f"contract block [{lo}, {hi}) is outside the batch's {contracts.rows} contracts"
        raise InputError(msg)
    sub, first, last = _ragged_slice(contracts.exercise.offsets, lo, hi)
    exercise = RaggedExerciseTimes(offsets=sub, times=np.ascontiguousarray(contracts.exercise.times[first:last]))
    cash = contracts.cash_dividends
    if cash is not None:
        sub, first, last = _ragged_slice(cash.offsets, lo, hi)
        cash = RaggedCashDividends(offsets=sub, times=np.ascontiguousarray(cash.times[first:last]),
                                   amounts=np.ascontiguousarray(cash.amounts[first:last]))

    def rows(v: np.ndarray | None) -> np.ndarray | None:
        return None if v is None else np.ascontiguousarray(v[lo:hi])

    return LsmRaggedContracts(
        initial_spots=rows(contracts.initial_spots), strikes=rows(contracts.strikes),
        maturities=rows(contracts.maturities), rates=rows(contracts.rates), volatilities=rows(contracts.volatilities),
        exercise=exercise, training_paths=rows(contracts.training_paths),
        evaluation_paths=rows(contracts.evaluation_paths), dividend_yields=rows(contracts.dividend_yields),
        cash_dividends=cash)


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
    return ("error", type(exc).__name__, message, row + row_offset if row >= 0 else -1,
            group + group_offset if group >= 0 else -1, int(getattr(exc, "code", 0)))


def _foreign(exc: BaseException, rank: int) -> tuple:
    """An exception outside the library's hierarchy, as a gathered outcome."""
    return ("error", "", f"shard on rank {rank} failed with {type(exc).__name__}: {exc}", -1, -1, 0)


def _process_group(process_group: object) -> tuple[object, int, int]:
    import torch.distributed as dist  # noqa: PLC0415 - only distributed callers need torch

    if not dist.is_available() or not dist.is_initialized():
        msg = "sharded LSM batches need an initialised torch.distributed process group"
        raise ExecutionError(msg)
    return dist, dist.get_rank(process_group), dist.get_world_size(process_group)


def _gather(dist: object, outcome: tuple, rank: int, world: int, process_group: object,
            local: BaseException | None) -> list:
    """Gathers every rank's outcome; raises the lowest rank's error, identically on every rank
    (chained to the original exception on the rank that raised it)."""
    gathered: list = [None] * world
    dist.all_gather_object(gathered, outcome, group=process_group)
    for i, entry in enumerate(gathered):
        if entry[0] == "error":
            _, kind, message, row, group, code = entry
            exc = _ERRORS.get(kind, ExecutionError)(message)
            exc.row, exc.group, exc.code = row, group, code  # type: ignore[attr-defined]
            raise exc from (local if i == rank else None)
    return gathered


def _frozen(values: object) -> np.ndarray:
    out = np.array(values, copy=True)  # a gathered copy arrives writeable
    out.flags.writeable = False
    return out


def _result_of(columns: tuple) -> LsmBatchResult:
    return LsmBatchResult(**{name: _frozen(v) for name, v in zip(_RESULT_COLUMNS, columns, strict=True)})


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
    dist, rank, world = _process_group(process_group)
    outcome: tuple | None = None
    local: BaseException | None = None
    lo = hi = row_lo = 0
    try:
        validate_lsm_call_grouped_batch(groups=groups, mesh=mesh, method=method)
        lo, hi = weighted_blocks(grouped_weights(groups, mesh, method), world)[rank]
        row_lo = int(groups.group_offsets[lo]) if hi > lo else 0
    except _LIBRARY_ERRORS as exc:
        outcome, local = _rebased(exc, 0, 0), exc
    except Exception as exc:  # noqa: BLE001 - every rank must reach the gather
        outcome, local = _foreign(exc, rank), exc
    if outcome is None:
        try:
            if hi > lo:
                block, block_mesh, block_method = shard_strike_groups(groups, mesh, method, lo, hi)
                part = pricer(groups=block, mesh=block_mesh, executor=executor, method=block_method)
                outcome = ("ok", tuple(getattr(part, name) for name in _RESULT_COLUMNS))
            else:
                outcome = ("empty",)
        except _LIBRARY_ERRORS as exc:
            outcome, local = _rebased(exc, row_lo, lo), exc
        except Exception as exc:  # noqa: BLE001 - every rank must reach the gather
            outcome, local = _foreign(exc, rank), exc
    gathered = _gather(dist, outcome, rank, world, process_group, local)
    return concatenate_results([_result_of(entry[1]) for entry in gathered if entry[0] == "ok"])


def price_lsm_call_ragged_sharded(  # noqa: PLR0913 - price_lsm_call_ragged's keywords
    *,
    contracts: LsmRaggedContracts,
    origin_exercise: OriginExercise,
    executor: object,
    training_stream: RandomStream,
    evaluation_stream: RandomStream,
    greeks: bool = False,
    process_group: object = None,
    pricer: Callable[..., object] | None = None,
    **method: object,
) -> LsmBatchResult | tuple[LsmBatchResult, LsmRaggedGreeks]:
    """Price a ragged batch (and, with greeks=True, its adjoint Greeks) across the ranks of the
    default (or given) process group; every rank passes the whole request and its own executor.
    `method` takes price_lsm_call_ragged's remaining keywords (insufficient_exercise_support, ...).
    `pricer` defaults to price_lsm_call_ragged or price_lsm_call_ragged_greeks."""
    dist, rank, world = _process_group(process_group)
    if pricer is None:
        pricer = price_lsm_call_ragged_greeks if greeks else price_lsm_call_ragged
    outcome: tuple | None = None
    local: BaseException | None = None
    lo = hi = 0
    try:
        validate_lsm_call_ragged(contracts=contracts, origin_exercise=origin_exercise, training_stream=training_stream,
                                 evaluation_stream=evaluation_stream, **method)
        lo, hi = weighted_blocks(ragged_weights(contracts), world)[rank]
    except _LIBRARY_ERRORS as exc:
        outcome, local = _rebased(exc, 0, 0), exc
    except Exception as exc:  # noqa: BLE001 - every rank must reach the gather
        outcome, local = _foreign(exc, rank), exc
    if outcome is None:
        try:
            if hi > lo:
                part = pricer(contracts=shard_ragged_contracts(contracts, lo, hi), origin_exercise=origin_exercise,
                              executor=executor, training_stream=_shifted(training_stream, lo),
                              evaluation_stream=_shifted(evaluation_stream, lo), **method)
                result, g = part if greeks else (part, None)
                sensitivities = None if g is None else (g.delta, g.vega, g.log_discount_sensitivities,
                                                        g.log_discount_offsets, g.dividend_sensitivities)
                outcome = ("ok", tuple(getattr(result, name) for name in _RESULT_COLUMNS), sensitivities)
            else:
                outcome = ("empty",)
        except _LIBRARY_ERRORS as exc:
            outcome, local = _rebased(exc, lo, lo), exc
        except Exception as exc:  # noqa: BLE001 - every rank must reach the gather
            outcome, local = _foreign(exc, rank), exc
    gathered = _gather(dist, outcome, rank, world, process_group, local)
    parts = [entry for entry in gathered if entry[0] == "ok"]
    result = concatenate_results([_result_of(entry[1]) for entry in parts])
    if not greeks:
        return result
    offsets, d_l, base = [np.zeros(1, dtype=np.int64)], [], 0
    for entry in parts:
        block_offsets = np.asarray(entry[2][3], dtype=np.int64)
        offsets.append(block_offsets[1:] + base)
        base += int(block_offsets[-1])
        d_l.append(np.asarray(entry[2][2]))
    return result, LsmRaggedGreeks(
        delta=_frozen(np.concatenate([e[2][0] for e in parts])), vega=_frozen(np.concatenate([e[2][1] for e in parts])),
        log_discount_sensitivities=_frozen(np.concatenate(d_l)), log_discount_offsets=_frozen(np.concatenate(offsets)),
        dividend_sensitivities=_frozen(np.concatenate([e[2][4] for e in parts])))


__all__ = [
    "concatenate_results",
    "group_block",
    "grouped_weights",
    "price_lsm_call_grouped_batch_sharded",
    "price_lsm_call_ragged_sharded",
    "ragged_weights",
    "shard_ragged_contracts",
    "shard_strike_groups",
    "weighted_blocks",
]
