"""The Arrow adapters (finoptions.arrow) on the host: zero-copy views of the Arrow buffers, the
buffer policy, and the schema / content checks of the reference's Polars adapter
(python/finoptions/polars.py), on pyarrow tables."""

from __future__ import annotations

import numpy as np
import pyarrow as pa
import pytest
from finoptions import DividendPolicy, EscrowedVolatilityConvention, MaturityBoundary
from finoptions.arrow import (
    ArrowAdapterTypeError,
    ArrowBufferError,
    ArrowContentError,
    ArrowSchemaError,
    BufferPolicy,
    CashDividendColumns,
    ContinuousYieldColumn,
    EscrowedCashDividendColumns,
    LsmCallColumns,
    LsmRaggedColumns,
    LsmStrikeGroupColumns,
    prepare_lsm_call_batch,
    prepare_lsm_ragged_contracts,
    prepare_lsm_strike_groups,
)
from finoptions.batch_lsm import CashDividendBatch, ContinuousDividendYieldBatch, EscrowedCashDividendBatch

COLUMNS = LsmCallColumns(initial_spot="s0", strike="k", maturity="t", rate="r", volatility="vol")
CASH = CashDividendColumns(times="div_t", amounts="div_a", policy=DividendPolicy.LIQUIDATOR,
                           maturity_boundary=MaturityBoundary.STRICTLY_BEFORE)


def call_table(rows: int = 6, *, large: bool = False) -> pa.Table:
    rng = np.random.default_rng(3)
    list_type = pa.large_list(pa.float64()) if large else pa.list_(pa.float64())
    times = [[0.25 * (j + 1) for j in range(i % 3)] for i in range(rows)]
    amounts = [[0.5 + j for j in range(i % 3)] for i in range(rows)]
    return pa.table({
        "s0": rng.uniform(80, 120, rows), "k": rng.uniform(80, 120, rows), "t": np.full(rows, 1.0),
        "r": np.full(rows, 0.03), "vol": np.full(rows, 0.2), "q": np.full(rows, 0.01),
        "div_t": pa.array(times, type=list_type), "div_a": pa.array(amounts, type=list_type),
    })


def buffer_address(column: pa.ChunkedArray | pa.Array) -> int:
    array = column.chunk(0) if isinstance(column, pa.ChunkedArray) else column
    return array.buffers()[1].address + array.offset * 8


def test_float64_columns_are_views_of_the_arrow_buffers() -> None:
    table = call_table()
    prepared = prepare_lsm_call_batch(table, columns=COLUMNS, dividends=ContinuousYieldColumn("q"))
    for name, values in (("s0", prepared.initial_spots), ("k", prepared.strikes), ("vol", prepared.volatilities)):
        assert values.ctypes.data == buffer_address(table.column(name))
        assert not values.flags.writeable
        np.testing.assert_array_equal(values, table.column(name).to_numpy())
    assert type(prepared.dividends) is ContinuousDividendYieldBatch
    assert prepared.dividends.annualized_decimals.ctypes.data == buffer_address(table.column("q"))
    assert prepared.rows == 6


@pytest.mark.parametrize("large", [False, True])
def test_cash_event_lists_keep_their_offsets_and_borrow_their_children(large) -> None:
    table = call_table(large=large)
    prepared = prepare_lsm_call_batch(table, columns=COLUMNS, dividends=CASH)
    assert type(prepared.dividends) is CashDividendBatch
    events = prepared.dividends.schedules
    times = table.column("div_t").chunk(0)
    assert events.offsets.tolist() == times.offsets.to_pylist()
    assert events.times.ctypes.data == times.values.buffers()[1].address
    assert events.times.tolist() == [v for row in times.to_pylist() for v in row]
    assert events.amounts.tolist() == [v for row in table.column("div_a").to_pylist() for v in row]
    escrowed = prepare_lsm_call_batch(table, columns=COLUMNS, dividends=EscrowedCashDividendColumns(
        times="div_t", amounts="div_a", volatility_convention=EscrowedVolatilityConvention.PREPAID_FORWARD,
        maturity_boundary=MaturityBoundary.STRICTLY_BEFORE))
    assert type(escrowed.dividends) is EscrowedCashDividendBatch


def test_a_sliced_table_keeps_the_lists_nonzero_offset_start() -> None:
    table = call_table(rows=9, large=True).slice(4, 4)
    prepared = prepare_lsm_call_batch(table, columns=COLUMNS, dividends=CASH)
    events = prepared.dividends.schedules
    assert events.offsets[0] > 0 and events.rows == 4
    assert events.times.tolist() == [v for row in table.column("div_t").to_pylist() for v in row]
    np.testing.assert_array_equal(prepared.initial_spots, table.column("s0").to_numpy())


def test_fragmented_columns_need_an_explicit_rechunk() -> None:
    table = pa.concat_tables([call_table(3), call_table(3)])
    with pytest.raises(ArrowBufferError, match="'s0' violates require_zero_copy: fragmented storage"):
        prepare_lsm_call_batch(table, columns=COLUMNS, dividends=CASH)
    prepared = prepare_lsm_call_batch(table, columns=COLUMNS, dividends=CASH,
                                      buffer_policy=BufferPolicy.ALLOW_RECHUNK)
    assert prepared.rows == 6 and prepared.dividends.schedules.rows == 6


def test_schema_and_content_violations_are_reported_without_values() -> None:
    table = call_table()
    with pytest.raises(ArrowSchemaError) as schema:
        prepare_lsm_call_batch(table.drop_columns(["k"]).append_column("k", pa.array(np.arange(6, dtype=np.int64))),
                               columns=COLUMNS, dividends=ContinuousYieldColumn("missing_q"))
    assert schema.value.missing == ("missing_q",)
    assert schema.value.mismatches == (("k", "float64", "int64"),)
    assert str(schema.value).startswith("invalid Arrow pricing schema: ")
    with_null = table.set_column(0, "s0", pa.array([1.0, None, 3.0, 4.0, 5.0, 6.0]))
    with pytest.raises(ArrowContentError, match=r"\('null_s0', 1\)"):
        prepare_lsm_call_batch(with_null, columns=COLUMNS, dividends=CASH)
    uneven = table.set_column(table.schema.get_field_index("div_a"), "div_a",
                              pa.array([[1.0]] * 6, type=pa.list_(pa.float64())))
    with pytest.raises(ArrowContentError, match="cash_event_length_mismatches"):
        prepare_lsm_call_batch(uneven, columns=COLUMNS, dividends=CASH)
    with pytest.raises(ArrowContentError, match="empty_frame"):
        prepare_lsm_call_batch(table.slice(0, 0), columns=COLUMNS, dividends=CASH)


def test_argument_types_and_column_names_are_strict() -> None:
    table = call_table()
    with pytest.raises(ArrowAdapterTypeError, match="frame must be a pyarrow.Table or pyarrow.RecordBatch"):
        prepare_lsm_call_batch(table.to_pandas(), columns=COLUMNS, dividends=CASH)
    with pytest.raises(ArrowAdapterTypeError, match="five distinct column names"):
        LsmCallColumns(initial_spot="a", strike="a", maturity="t", rate="r", volatility="v")
    with pytest.raises(ArrowAdapterTypeError, match="nonempty plain string"):
        ContinuousYieldColumn("")
    with pytest.raises(ArrowAdapterTypeError, match="distinct contract and dividend columns"):
        prepare_lsm_call_batch(table, columns=COLUMNS, dividends=ContinuousYieldColumn("s0"))
    with pytest.raises(ArrowAdapterTypeError, match="buffer_policy must be BufferPolicy"):
        prepare_lsm_call_batch(table, columns=COLUMNS, dividends=CASH, buffer_policy="allow_rechunk")
    batch = table.to_batches()[0]
    assert prepare_lsm_call_batch(batch, columns=COLUMNS, dividends=CASH).rows == 6


STATES = LsmStrikeGroupColumns(initial_spot="s0", maturity="t", rate="r", volatility="vol")


def test_strike_groups_borrow_three_axes() -> None:
    states = call_table(4)
    strikes = pa.table({"k": np.linspace(80, 120, 10)})
    offsets = pa.array([0, 2, 5, 9, 10], type=pa.uint32())
    prepared = prepare_lsm_strike_groups(states, strikes, group_offsets=offsets, state_columns=STATES,
                                         strike_column="k", dividends=CASH)
    native = prepared.native
    assert prepared.group_count == 4 and prepared.rows == 10
    assert native.group_offsets.ctypes.data == offsets.buffers()[1].address
    assert native.strikes.ctypes.data == buffer_address(strikes.column("k"))
    assert native.initial_spots.ctypes.data == buffer_address(states.column("s0"))
    assert native.dividends.schedules.rows == 4


def test_strike_group_offsets_are_checked() -> None:
    states, strikes = call_table(4), pa.table({"k": np.linspace(80, 120, 10)})

    def prepare(offsets):
        return prepare_lsm_strike_groups(states, strikes, group_offsets=offsets, state_columns=STATES,
                                         strike_column="k", dividends=CASH)

    with pytest.raises(ArrowSchemaError, match="group_offsets"):
        prepare(pa.array([0, 2, 5, 9, 10], type=pa.int64()))
    with pytest.raises(ArrowContentError) as content:
        prepare(pa.array([0, 5, 5, 9], type=pa.uint32()))
    assert content.value.violations == (("group_offset_count_mismatch", 1), ("group_offset_boundary_mismatch", 1),
                                        ("empty_or_reversed_groups", 1))
    with pytest.raises(ArrowContentError, match="empty_strike_frame"):
        prepare_lsm_strike_groups(states, strikes.slice(0, 0), group_offsets=pa.array([0], type=pa.uint32()),
                                  state_columns=STATES, strike_column="k", dividends=CASH)


def test_ragged_contracts_carry_per_row_paths_and_exercise_lists() -> None:
    rows = 5
    table = call_table(rows, large=True).append_column(
        "train", pa.array(np.arange(1, rows + 1, dtype=np.uint64) * 1000)).append_column(
        "eval", pa.array(np.arange(1, rows + 1, dtype=np.uint64) * 2000)).append_column(
        "ex", pa.array([[0.1 * (j + 1) for j in range(i + 1)] for i in range(rows)], type=pa.large_list(pa.float64())))
    columns = LsmRaggedColumns(initial_spot="s0", strike="k", maturity="t", rate="r", volatility="vol",
                               training_paths="train", evaluation_paths="eval", exercise_times="ex",
                               dividend_yield="q")
    contracts = prepare_lsm_ragged_contracts(table, columns=columns, cash_dividends=("div_t", "div_a"))
    assert contracts.rows == rows
    assert contracts.training_paths.tolist() == [1000, 2000, 3000, 4000, 5000]
    assert contracts.training_paths.ctypes.data == buffer_address(table.column("train"))
    assert contracts.exercise.offsets.tolist() == [0, 1, 3, 6, 10, 15]
    assert contracts.cash_dividends.rows == rows and contracts.dividend_yields is not None
    with pytest.raises(ArrowSchemaError, match="train"):
        prepare_lsm_ragged_contracts(table.set_column(table.schema.get_field_index("train"), "train",
                                                      pa.array(np.arange(rows, dtype=np.int64))),
                                     columns=columns)
