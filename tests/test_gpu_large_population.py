"""Training populations beyond the on-chip backward pass (fo_price_lsm_call_f64 / price_lsm_call).

Up to 148 SMs x 1024 threads x 9 paths the backward pass keeps every path's value and spots in
shared memory; above that it keeps the values in HBM and reads the spots from the stored rows, so a
single contract takes any path count the device memory holds (the reference accepts up to
2^32 - 1 paths per random domain, crates/finoptions-sim/src/path/seeded.rs:391-394). Prices, SE,
stopping counts and diagnostics must match the oracle as for any other population.
"""

from __future__ import annotations

import ctypes
import os

import _oracle
import pytest
from _workloads import weekly_call_kwargs
from finoptions import _abi
from finoptions._requests import lsm_call_request, lsm_call_result

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))


def gpu_price(native_executor, kwargs: dict) -> tuple:
    req = lsm_call_request(**kwargs)
    res = lsm_call_result(req.exercise_rows)
    err = _abi.FoError()
    assert _abi.load().fo_price_lsm_call_f64(native_executor.raw, ctypes.byref(req.struct), ctypes.byref(res.struct),
                                             ctypes.byref(err)) == 0, err.message
    return res.as_tuple()


def assert_matches_oracle(gpu: tuple, want: tuple) -> None:
    price, paths, sd, se, nodes, counts, diags = want
    assert gpu[0] == pytest.approx(price, rel=1e-9)
    assert gpu[2] == pytest.approx(sd, rel=1e-9)
    assert gpu[3] == pytest.approx(se, rel=1e-9)
    assert (gpu[1], gpu[4], gpu[5]) == (paths, nodes, counts)
    for d, o in zip(gpu[6], diags, strict=True):
        assert d[:2] == o[:2]
        if d[1] == "origin_decision":  # (node, kind, exercised, continuation value, None)
            assert d[2] == o[2] and d[3] == pytest.approx(o[3], rel=1e-9)
        else:  # node, kind, in-the-money counts, columns
            assert d[:5] == o[:5]


def test_weekly_contract_at_2p21_paths_matches_the_oracle(native_executor) -> None:
    kwargs = weekly_call_kwargs(1 << 21)
    assert_matches_oracle(gpu_price(native_executor, kwargs), _oracle.price_lsm_call(lsm_call_request(**kwargs), THREADS))


@pytest.mark.parametrize("paths", [1_400_003, 3_000_000])
def test_ragged_large_populations_match_the_oracle(native_executor, paths: int) -> None:
    """Path counts that fill the last paths-per-thread round only partly, on a short schedule with a
    cash dividend and the origin decision."""
    kwargs = weekly_call_kwargs(paths)
    t = [i / 6 for i in range(7)]
    kwargs.update(schedule_times=t, curve_times=t, log_discounts=[-0.05 * v for v in t], dividend_yield_times=t,
                  cumulative_dividend_yields=[0.0] * 7, dividend_nodes=[3], dividend_amounts=[2.0],
                  exercise_nodes=[0, 1, 2, 3, 4, 5], expiry_node=6, training_domain=5, evaluation_domain=6)
    kwargs["log_discounts"][0] = 0.0
    assert_matches_oracle(gpu_price(native_executor, kwargs), _oracle.price_lsm_call(lsm_call_request(**kwargs), THREADS))
