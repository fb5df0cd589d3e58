"""The allocation-free pricing entry point, through the C ABI.

fo_price_lsm_call_f64_noalloc serves callers that cannot allocate device memory (their device
memory belongs to another allocator, or cudaMalloc's implicit synchronisation is not acceptable on
their path). It must produce the same result as fo_price_lsm_call_f64 on consecutive calls, which
share its one device scratch array, must leave the device's free memory unchanged, and must reject
requests larger than that array.
"""

from __future__ import annotations

import ctypes
import math

import pytest
from finoptions import _abi
from finoptions._requests import lsm_call_request, lsm_call_result

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def weekly_request(paths: int, dividends=((13, 1.5), (39, 1.5))):
    steps = 52
    t = [i / steps for i in range(steps + 1)]
    return lsm_call_request(
        initial_spot=100.0, strike=100.0, schedule_times=t, curve_times=t,
        log_discounts=[0.0 if i == 0 else -0.04 * t[i] for i in range(steps + 1)], dividend_yield_times=t,
        cumulative_dividend_yields=[0.0 if i == 0 else 0.02 * t[i] for i in range(steps + 1)],
        dividend_nodes=[d[0] for d in dividends], dividend_amounts=[d[1] for d in dividends],
        exercise_nodes=list(range(steps)), expiry_node=steps, annualized_volatility=0.25, dividend_policy=0,
        training_paths=paths, evaluation_paths=paths, training_seed=11, training_domain=1, evaluation_seed=11,
        evaluation_domain=2, polynomial_degree=4, rank_tolerance=1e-12, condition_limit=1e8, tie_rule=0,
        insufficient_exercise_support=0,
    )


def price_no_alloc(request):
    result = lsm_call_result(request.exercise_rows)
    err = _abi.FoError()
    status = _abi.load().fo_price_lsm_call_f64_noalloc(ctypes.byref(request.struct), None, ctypes.byref(result.struct),
                                                       ctypes.byref(err))
    return status, err, (result.as_tuple() if status == 0 else None)


def test_no_alloc_entry_matches_the_allocating_entry_on_consecutive_calls(native_executor) -> None:
    request = weekly_request(65536)
    result = lsm_call_result(request.exercise_rows)
    err = _abi.FoError()
    assert _abi.load().fo_price_lsm_call_f64(native_executor.raw, ctypes.byref(request.struct),
                                             ctypes.byref(result.struct), ctypes.byref(err)) == 0, err.message
    expected = result.as_tuple()
    for _ in range(2):
        status, err, got = price_no_alloc(request)
        assert status == 0, err.message
        price, paths, sd, se, nodes, counts, diagnostics = got
        assert (paths, nodes, counts) == (expected[1], expected[4], expected[5])
        assert math.isclose(price, expected[0], rel_tol=RTOL)
        assert math.isclose(sd, expected[2], rel_tol=RTOL)
        assert math.isclose(se, expected[3], rel_tol=RTOL)
        assert [d[:8] for d in diagnostics] == [d[:8] for d in expected[6]]
        for d, e in zip(diagnostics, expected[6], strict=True):
            for a, b in zip(d[8:], e[8:], strict=True):
                assert (a is None and b is None) or math.isclose(a, b, rel_tol=RTOL)


def test_no_alloc_entry_rejects_requests_beyond_its_scratch() -> None:
    status, err, _ = price_no_alloc(weekly_request(1 << 20))
    assert status == _abi.FO_ERR_EXECUTION
    message = err.message.decode()
    assert "allocation-free entry point holds at most 67108864 bytes" in message


def test_no_alloc_calls_leave_the_device_free_memory_unchanged() -> None:
    """After a first call (which loads the kernels it launches), further calls whose scratch needs
    (about 28 MB here) are well above the driver's allocation granularity move no device memory."""
    import torch

    torch.cuda.mem_get_info(0)  # the runtime's own set-up happens before anything is measured
    request = weekly_request(65536)
    status, err, _ = price_no_alloc(request)
    assert status == 0, err.message
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        status, err, _ = price_no_alloc(request)
        assert status == 0, err.message
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before
