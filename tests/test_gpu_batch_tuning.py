"""Launch shapes of the persistent batch launch and the autotuner (fo_executor_set_batch_tuning).

A batch wave runs as one persistent launch whose CTAs take work items from a queue. Its shape
(blocks per simulation / evaluation item, strikes per evaluation item, CTAs per SM) changes only how
the work is cut and scheduled: every shape must give the same twelve columns and the same Greeks,
bit for bit, and the default shape must match the oracle. With the autotuner on, the first wave of
a class times candidate shapes and later waves of the class reuse the chosen one.
"""

from __future__ import annotations

import ctypes

import _oracle
import numpy as np
import pytest
from _workloads import grouped_columns, grouped_request, ragged_columns, ragged_request, ragged_row_as_call
from finoptions import _abi
from finoptions._requests import batch_columns
from test_gpu_batch import assert_columns, gpu_batch

pytestmark = pytest.mark.gpu

# (simulation blocks per item, evaluation blocks per item, strikes per evaluation item, CTAs per SM,
# phases): one persistent launch (phases 0) or the phase kernels (phases 1).
SHAPES = [(2, 1, 8, 0, 0), (1, 1, 8, 0, 0), (8, 4, 8, 0, 0), (2, 2, 4, 0, 0), (2, 1, 2, 2, 0), (1, 4, 1, 1, 0),
          (2, 1, 8, 0, 1), (4, 2, 4, 0, 1)]


def set_shape(native_executor, shape) -> None:
    tuning = _abi.FoBatchTuning(*shape)
    err = _abi.FoError()
    assert _abi.load().fo_executor_set_batch_tuning(native_executor.raw, 0, ctypes.byref(tuning),
                                                    ctypes.byref(err)) == 0, err.message


def autotune(native_executor) -> None:
    err = _abi.FoError()
    assert _abi.load().fo_executor_set_batch_tuning(native_executor.raw, 1, None, ctypes.byref(err)) == 0


def launch_info(native_executor) -> _abi.FoBatchLaunchInfo:
    info = _abi.FoBatchLaunchInfo()
    assert _abi.load().fo_executor_batch_launch(native_executor.raw, ctypes.byref(info)) == 0
    return info


def ragged_greeks(native_executor, c):
    nodes = sum(len(ragged_row_as_call(c, r)["schedule_times"]) for r in range(c.rows))
    arrays = {"delta": np.zeros(c.rows), "vega": np.zeros(c.rows), "d_l": np.zeros(nodes),
              "offsets": np.zeros(c.rows + 1, dtype=np.int64), "d_d": np.zeros(max(c.dividend_times.size, 1))}
    g = _abi.FoRaggedGreeksColumns()
    dp = ctypes.POINTER(ctypes.c_double)
    g.delta, g.vega = arrays["delta"].ctypes.data_as(dp), arrays["vega"].ctypes.data_as(dp)
    g.log_discount_sensitivities = arrays["d_l"].ctypes.data_as(dp)
    g.log_discount_capacity = nodes
    g.log_discount_offsets = arrays["offsets"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    g.dividend_sensitivities = arrays["d_d"].ctypes.data_as(dp)
    req = ragged_request(c)
    cols = batch_columns(req.rows)
    err = _abi.FoError()
    assert _abi.load().fo_price_lsm_ragged_f64(native_executor.raw, ctypes.byref(req.struct), ctypes.byref(cols.struct),
                                               ctypes.byref(g), ctypes.byref(err)) == 0, err.message
    return cols.as_tuple(), arrays


@pytest.fixture
def fixed_shapes(native_executor):
    yield
    autotune(native_executor)  # the session executor goes back to the default


def test_every_launch_shape_prices_a_grouped_batch_identically(native_executor, fixed_shapes) -> None:
    c = grouped_columns(12, 8, seed=71, min_exercise=6, max_exercise=20)
    req = grouped_request(c, 4096)
    results = []
    for shape in SHAPES:
        set_shape(native_executor, shape)
        status, err, out = gpu_batch(native_executor, req)
        assert status == 0, err.message
        info = launch_info(native_executor)
        assert info.source == 0 and info.tuning.sim_blocks == shape[0] and info.tuning.eval_blocks == shape[1]
        assert info.tuning.strikes == shape[2] and info.tuning.phases == shape[4] and info.grid > 0 and info.items > 0
        results.append(out)
    for out in results[1:]:
        for got, want in zip(out, results[0], strict=True):
            np.testing.assert_array_equal(got, want)
    assert_columns(results[0], _oracle.price_lsm_grouped(req, 16))


def test_every_launch_shape_gives_the_same_ragged_greeks(native_executor, fixed_shapes) -> None:
    # Up to 120,000 paths: the larger rows are fitted by teams of up to four CTAs.
    c = ragged_columns(9, seed=73, min_paths=1500, max_paths=120_000, min_exercise=4, max_exercise=24)
    results = []
    for shape in SHAPES:
        set_shape(native_executor, shape)
        results.append(ragged_greeks(native_executor, c))
    for cols, arrays in results[1:]:
        for got, want in zip(cols, results[0][0], strict=True):
            np.testing.assert_array_equal(got, want)
        for name, values in arrays.items():
            np.testing.assert_array_equal(values, results[0][1][name], err_msg=name)


def test_the_autotuner_tunes_a_class_once_and_reuses_its_shape(native_executor) -> None:
    autotune(native_executor)
    c = grouped_columns(10, 8, seed=79, min_exercise=6, max_exercise=14)
    req = grouped_request(c, 2048 + 77)  # a path count no other test uses: a new class
    status, err, first = gpu_batch(native_executor, req)
    assert status == 0, err.message
    info = launch_info(native_executor)
    assert info.source == 2 and info.tuning_launches >= 5
    status, err, second = gpu_batch(native_executor, req)
    assert status == 0, err.message
    again = launch_info(native_executor)
    assert again.source == 1
    assert (again.tuning.sim_blocks, again.tuning.eval_blocks, again.tuning.ctas_per_sm) == (
        info.tuning.sim_blocks, info.tuning.eval_blocks, info.tuning.ctas_per_sm)
    for got, want in zip(second, first, strict=True):
        np.testing.assert_array_equal(got, want)
    assert_columns(first, _oracle.price_lsm_grouped(req, 16))


def test_launch_shapes_outside_their_range_are_rejected(native_executor, fixed_shapes) -> None:
    for shape in ((0, 1, 8, 0, 0), (2, 65, 8, 0, 0), (2, 1, 3, 0, 0), (2, 1, 8, 9, 0), (2, 1, 8, 0, 2)):
        tuning = _abi.FoBatchTuning(*shape)
        err = _abi.FoError()
        assert _abi.load().fo_executor_set_batch_tuning(native_executor.raw, 0, ctypes.byref(tuning),
                                                        ctypes.byref(err)) == _abi.FO_ERR_EXECUTION
        assert "outside its range" in err.message.decode()


def test_a_repeated_wave_replays_its_captured_graph(native_executor, fixed_shapes) -> None:
    """A wave is captured as a CUDA graph once per launch key; the same request again replays it, and
    a different request captures anew. Replays give the same columns."""
    set_shape(native_executor, (2, 1, 8, 0, 1))
    c = grouped_columns(7, 8, seed=83, min_exercise=5, max_exercise=11)
    req = grouped_request(c, 3000)
    outs = []
    for expected in ((0, 1), (1, 0), (1, 0)):
        status, err, out = gpu_batch(native_executor, req)
        assert status == 0, err.message
        info = launch_info(native_executor)
        assert (info.graph_replays, info.graph_captures) == expected
        outs.append(out)
    for out in outs[1:]:
        for got, want in zip(out, outs[0], strict=True):
            np.testing.assert_array_equal(got, want)
    status, err, _ = gpu_batch(native_executor, grouped_request(c, 3001))
    assert status == 0, err.message
    assert (launch_info(native_executor).graph_replays, launch_info(native_executor).graph_captures) == (0, 1)
    assert_columns(outs[0], _oracle.price_lsm_grouped(req, 16))
