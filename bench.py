#!/usr/bin/env python
"""LSM path-steps/s on one B200: the 52-node weekly single-contract workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--paths P]

Workload (one "step" = pricing one contract end to end: training simulation, backward policy fit,
independent evaluation): S0 = K = 100, T = 1, 53-node weekly grid t_i = i/52, exercise at nodes
0..51 (the origin is a common decision) plus expiry 52, log-discounts -0.04 t, cumulative
continuous yield 0.02 t, sigma = 0.25, 2^20 training + 2^20 evaluation paths (Philox seed 11,
domains 1 / 2), degree-4 regression, rank tolerance 1e-12, condition limit 1e8, strictly-greater
ties, insufficient support = fail. path-steps per step = (2^20 + 2^20) * 52 intervals. `--paths`
shrinks both populations for small profiler captures; the headline run keeps 2^20.

`value` is timed on the device (CUDA events around K launches of a resident plan); `e2e` is the
same metric through the public API finoptions.price_lsm_call with host inputs and host results.
Multi-GPU runs are independent replicas (a single contract does not shard): value = all ranks'
path-steps / max-over-ranks time. `--impl reference` times the CPU restatement of the reference
engine on the host cores on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "finoptions-engine_b200"))
sys.path.insert(0, str(ROOT / "tests"))

STEPS_IN_GRID = 52
PATHS = 1 << 20
METRIC = "lsm_path_steps_per_s"
UNIT = "path-steps/s"
KERNEL_NAMES = ("simulate_kernel", "backward_kernel", "diagnose_kernel", "evaluate_kernel", "finalize_kernel")


def workload_kwargs(paths: int = PATHS) -> dict:
    import _workloads

    return _workloads.weekly_call_kwargs(paths)


def path_steps(paths: int = PATHS) -> int:
    return 2 * paths * STEPS_IN_GRID


def config(paths: int = PATHS) -> dict:
    return {
        "workload": "weekly single-contract LSM call: S0=K=100, T=1, 52 weekly intervals, exercise nodes 0..51 + expiry",
        "contract": "r=0.04 (log-discount -r t), continuous yield q=0.02, sigma=0.25, degree 4",
        "training_paths": paths,
        "evaluation_paths": paths,
        "streams": "Philox seed 11, domains 1 (training) / 2 (evaluation)",
        "global_batch": 1,
        "path_steps_per_step": path_steps(paths),
        "parallelism": "replicas",
        "l2": f"working set vs L2: {8 * STEPS_IN_GRID * paths / 1e6:.0f} MB of stored training rows per step, 126 MB L2",
    }


# ---- helpers -----------------------------------------------------------------------------------


def dist_info() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """Samples SM clocks and throttle reasons through NVML while the timed region runs."""

    REASONS = {
        "gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4, "hw_slowdown": 0x8,
        "sync_boost": 0x10, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "hw_power_brake_slowdown": 0x80, "display_clock_setting": 0x100,
    }

    def __init__(self, device: int, period: float = 0.05) -> None:
        self.device = device
        self.period = period
        self.samples: list[int] = []
        self.reasons: set[str] = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nvml = pynvml
            self._handle = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._handle, pynvml.NVML_CLOCK_SM)
        except Exception:  # noqa: BLE001 - clocks are reported as unavailable
            self._nvml = None

    def sample(self) -> None:
        if self._nvml is None:
            return
        nv = self._nvml
        self.samples.append(nv.nvmlDeviceGetClockInfo(self._handle, nv.NVML_CLOCK_SM))
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self._handle)
        for name, bit in self.REASONS.items():
            if mask & bit and name != "gpu_idle":
                self.reasons.add(name)

    def _run(self) -> None:
        while not self._stop.is_set():
            self.sample()
            self._stop.wait(self.period)

    def __enter__(self) -> ClockSampler:
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc: object) -> None:
        self._stop.set()
        if self._thread:
            self._thread.join()

    def report(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def measured_peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.is_file():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel: str) -> float | None:
    """DRAM bytes per stored path-row for `kernel` from the committed ncu summary, if present."""
    path = ROOT / "profiles" / "traffic.json"
    if not path.is_file():
        return None
    data = json.loads(path.read_text())
    entry = data.get(kernel)
    return None if entry is None else float(entry["dram_bytes_per_path_row"])


def profiled_instructions(kernel: str) -> float | None:
    """Warp instructions per path-step of `kernel` from the committed ncu summary, if present."""
    path = ROOT / "profiles" / "issue.json"
    if not path.is_file():
        return None
    data = json.loads(path.read_text())
    entry = data.get(kernel)
    return None if entry is None else float(entry["warp_instructions"]) / float(data["path_steps_profiled"])


def issue_rate(kernel: str, ms: float, path_steps_per_launch: int, sm_mhz: float, sms: int) -> dict | None:
    """Issue-rate roofline of an instruction-bound kernel: warp instructions per launch (the profiled
    count per path-step times the launch's path-steps) over its measured time, against the issue
    peak of one warp instruction per scheduler per cycle (4 per SM) at the SM clock seen under load."""
    per_step = profiled_instructions(kernel)
    if per_step is None or ms <= 0 or sm_mhz <= 0:
        return None
    achieved = per_step * path_steps_per_launch / (ms / 1e3)
    peak = 4.0 * sms * sm_mhz * 1e6
    return {"warp_instructions_per_path_step": round(per_step, 2), "achieved_winst_per_s": achieved,
            "peak_winst_per_s": peak, "frac": round(achieved / peak, 4)}


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def oracle_price(kwargs: dict, threads: int) -> tuple:
    import _oracle
    from finoptions._requests import lsm_call_request

    return _oracle.price_lsm_call(lsm_call_request(**kwargs), threads)


def public_call_arguments(kw: dict, executor) -> dict:
    """finoptions.price_lsm_call's arguments for a contract given as single-contract kwargs."""
    import finoptions as fo

    times = tuple(kw["schedule_times"])
    schedule = fo.EventSchedule(
        times=times,
        dividends=tuple(fo.CashDividend(node=int(n), amount=float(a))
                        for n, a in zip(kw["dividend_nodes"], kw["dividend_amounts"], strict=True)),
        exercise_nodes=tuple(int(n) for n in kw["exercise_nodes"]), expiry_node=int(kw["expiry_node"]))
    support = (fo.InsufficientExerciseSupportPolicy.CONTINUE if kw["insufficient_exercise_support"]
               else fo.InsufficientExerciseSupportPolicy.FAIL)
    return dict(
        initial_spot=float(kw["initial_spot"]), strike=float(kw["strike"]), schedule=schedule,
        curve=fo.LogDiscountCurve(times=times, log_discounts=tuple(float(v) for v in kw["log_discounts"])),
        dividend_yield_curve=fo.CumulativeDividendYieldCurve(
            times=times, cumulative_yields=tuple(float(v) for v in kw["cumulative_dividend_yields"])),
        volatility=fo.ConstantVolatility(float(kw["annualized_volatility"])),
        dividend_policy=fo.DividendPolicy.LIQUIDATOR, executor=executor,
        method=fo.Lsm(training_paths=int(kw["training_paths"]), evaluation_paths=int(kw["evaluation_paths"]),
                      training_stream=fo.RandomStream(seed=int(kw["training_seed"]), domain=int(kw["training_domain"])),
                      evaluation_stream=fo.RandomStream(seed=int(kw["evaluation_seed"]),
                                                        domain=int(kw["evaluation_domain"])),
                      insufficient_exercise_support=support))


def one_by_one(calls: list[dict], batch_prices, batch_errors) -> dict:
    """Prices the contracts one call at a time through finoptions.price_lsm_call (host inputs, host
    results, every call synchronous) and checks each against its batch row: the same populations,
    so the same price and standard error."""
    import finoptions as fo
    import numpy as np

    fo.price_lsm_call(**calls[0])
    t0 = time.perf_counter()
    results = [fo.price_lsm_call(**a) for a in calls]
    wall = time.perf_counter() - t0
    prices = np.array([r.price for r in results])
    errors = np.array([r.standard_error for r in results])
    return {"contracts": len(calls), "seconds": wall, "contracts_per_s": len(calls) / wall,
            "api": "finoptions.price_lsm_call(executor=CudaExecutor), one contract per call",
            "max_rel_price_difference_vs_batch": relative_difference(prices, batch_prices),
            "max_rel_se_difference_vs_batch": relative_difference(errors, batch_errors)}


def relative_difference(a, b) -> float:
    """Largest |a - b| / |b| over the entries, with 0 where both are 0 (worthless contracts)."""
    import numpy as np

    diff = np.abs(np.asarray(a) - np.asarray(b))
    scale = np.abs(np.asarray(b))
    return float(np.max(np.where(diff == 0.0, 0.0, diff / np.where(scale == 0.0, 1.0, scale))))


# ---- our arm -----------------------------------------------------------------------------------


def run_ours(args: argparse.Namespace) -> dict | None:
    import torch

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from finoptions import _abi
    from finoptions._native import CudaExecutor
    from finoptions._requests import lsm_call_request, lsm_call_result

    lib = _abi.load()
    executor = CudaExecutor(local)
    paths = args.paths
    kwargs = workload_kwargs(paths)
    request = lsm_call_request(**kwargs)
    err = _abi.FoError()
    plan = ctypes.c_void_p()
    status = lib.fo_lsm_call_plan_create(executor.raw, ctypes.byref(request.struct), ctypes.byref(plan), ctypes.byref(err))
    if status:
        raise RuntimeError(err.message.decode())
    kernels = ctypes.c_uint64()
    lib.fo_lsm_call_plan_kernel_count(plan, ctypes.byref(kernels))
    h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
    lib.fo_lsm_call_plan_transfer_bytes(plan, ctypes.byref(h2d), ctypes.byref(d2h))
    elapsed = ctypes.c_double()
    kernel_ms = (ctypes.c_double * 8)()

    def timed(iterations: int, per_kernel: bool) -> float:
        st = lib.fo_lsm_call_plan_time_launches(plan, iterations, ctypes.byref(elapsed),
                                                kernel_ms if per_kernel else None, 8, ctypes.byref(err))
        if st:
            raise RuntimeError(err.message.decode())
        return elapsed.value

    timed(args.warmup, False)
    # Device-timed region: K launches between CUDA events on the plan's stream.
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with clocks:
        device_ms = timed(args.steps, False)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
        t = torch.tensor([device_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        device_ms = float(t.item())
    # Per-kernel device times (separate pass with events between kernels).
    timed(max(1, min(args.steps, 20)), True)
    per_kernel = {KERNEL_NAMES[k]: kernel_ms[k] for k in range(int(kernels.value))}
    per_kernel_launches = max(1, min(args.steps, 20))
    result = lsm_call_result(request.exercise_rows)
    st = lib.fo_lsm_call_plan_collect(plan, ctypes.byref(result.struct), ctypes.byref(err))
    if st:
        raise RuntimeError(err.message.decode())
    price, _, _, se, *_ = result.as_tuple()
    lib.fo_lsm_call_plan_destroy(plan)

    # End to end through the public API: host inputs in, host results out, every step.
    import finoptions as fo

    times = tuple(kwargs["schedule_times"])
    schedule = fo.EventSchedule(times=times, dividends=(), exercise_nodes=tuple(kwargs["exercise_nodes"]),
                                expiry_node=kwargs["expiry_node"])
    api_args = dict(
        initial_spot=kwargs["initial_spot"], strike=kwargs["strike"], schedule=schedule,
        curve=fo.LogDiscountCurve(times=times, log_discounts=tuple(kwargs["log_discounts"])),
        dividend_yield_curve=fo.CumulativeDividendYieldCurve(times=times,
                                                             cumulative_yields=tuple(kwargs["cumulative_dividend_yields"])),
        volatility=fo.ConstantVolatility(kwargs["annualized_volatility"]),
        dividend_policy=fo.DividendPolicy.LIQUIDATOR, executor=fo.CudaExecutor(device=local),
        method=fo.Lsm(training_paths=paths, evaluation_paths=paths, training_stream=fo.RandomStream(seed=11, domain=1),
                      evaluation_stream=fo.RandomStream(seed=11, domain=2),
                      insufficient_exercise_support=fo.InsufficientExerciseSupportPolicy.FAIL),
    )
    for _ in range(args.warmup):
        fo.price_lsm_call(**api_args)
    e2e_steps = max(1, min(args.steps, 100))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        api_result = fo.price_lsm_call(**api_args)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
    if api_result.price != price:
        raise RuntimeError("public API and resident plan disagree")
    if rank != 0:
        return None

    ms_per_step = device_ms / args.steps
    value = world * path_steps(paths) * args.steps / (device_ms / 1e3)
    # Roofline of the dominant path-data kernel: stored rows are written once (simulate) and read
    # once (backward); algorithmic bytes = 8 B per stored path-row.
    stored_rows = STEPS_IN_GRID  # rows 1..52 (the origin row is the constant S0, never stored)
    algorithmic = 8 * stored_rows * paths
    hbm_peak, peak_kind = measured_peaks()
    roofline_all = {}
    # The diagnostic runs on a side stream beside the evaluation: it is timed on its own stream
    # and left out of the shares of the serial kernel chain.
    serial_ms = sum(v for k, v in per_kernel.items() if k != "diagnose_kernel")
    for name in KERNEL_NAMES[: int(kernels.value)]:
        ms = per_kernel[name] / per_kernel_launches
        bytes_per_launch = algorithmic if name in ("simulate_kernel", "backward_kernel") else 0
        roofline_all[name] = {
            "ms_per_launch": round(ms, 4),
            "share": None if name == "diagnose_kernel" else round(per_kernel[name] / serial_ms, 4),
            "algorithmic_bytes": bytes_per_launch,
            "achieved_gbs": round(bytes_per_launch / (ms / 1e3) / 1e9, 1) if bytes_per_launch else 0.0,
        }
        if name == "diagnose_kernel":
            roofline_all[name]["concurrent_with"] = "evaluate_kernel"
    dominant = max(("simulate_kernel", "backward_kernel"), key=lambda k: per_kernel[k])
    dom_ms = per_kernel[dominant] / per_kernel_launches
    achieved = algorithmic / (dom_ms / 1e3) / 1e9
    traffic_unit = profiled_traffic(dominant)
    clock_report = clocks.report()
    sm_mhz = float(clock_report.get("sm_mhz") or 0.0)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for name in ("simulate_kernel", "evaluate_kernel"):
        rate = issue_rate(name, roofline_all[name]["ms_per_launch"], path_steps(paths) // 2, sm_mhz, sms)
        if rate is not None:
            roofline_all[name]["issue"] = rate
    out = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Philox paths of the configured contract)",
        "config": dict(config(paths), contracts_per_s=world * args.steps / (device_ms / 1e3)),
        "e2e": {
            "value": world * path_steps(paths) * e2e_steps / e2e_s,
            "unit": UNIT,
            "h2d_bytes_per_step": int(h2d.value),
            "d2h_bytes_per_step": int(d2h.value),
            "api": "finoptions.price_lsm_call(executor=CudaExecutor)",
        },
        "gpu_launches": int(kernels.value) * args.steps,
        "roofline": {
            "kernel": dominant,
            # The backward pass is bound by the latency of its 52 dependent row exchanges (each row
            # a grid-wide reduction and a regression solve), not by HBM: achieved / peak below is its
            # HBM fraction, us_per_row the figure that bounds it.
            "bound": "latency" if dominant == "backward_kernel" else "hbm",
            "achieved": round(achieved, 1),
            "peak": hbm_peak,
            "peak_source": peak_kind,
            "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 4),
            "traffic": None if traffic_unit is None else int(traffic_unit * stored_rows * paths),
            "rows": stored_rows,
            "us_per_row": round(dom_ms * 1e3 / stored_rows, 2),
        },
        "kernels": roofline_all,
        "clocks": clock_report,
        "result": {"price": price, "standard_error": se},
    }
    if world == 1:
        out["cpu_baseline"] = cpu_baseline(paths)
    else:
        # The batch, Greeks and ragged sections are single-GPU measurements, reported at N = 1;
        # the other ranks have left, so the multi-GPU line carries the replicated contract only.
        args.skip_batched = args.skip_greeks = args.skip_ragged = True
    if not args.skip_batched:
        out["batched"] = run_grouped(args, executor)
    if not args.skip_greeks:
        out["greeks"] = run_greeks(args, executor)
    if not args.skip_ragged:
        out["ragged"] = run_ragged(args, executor)
    return out


# ---- ragged batch with per-contract path counts + Greeks -----------------------------------------

RAGGED_CONTRACTS = 1024
RAGGED_SAMPLE = 16


def run_ragged(args: argparse.Namespace, executor) -> dict:
    """1024 independent contracts, path counts log-uniform in [8192, 262144] (same per role), 4-104
    exercise dates, half continuous yield / half 1-6 cash dividends, seed 41: one batch call priced
    alone and with the adjoint Greeks (delta, vega, dP/dL per mesh node, dP/dD per cash event)."""
    import _oracle
    import _workloads
    import numpy as np
    from finoptions import _abi
    from finoptions._requests import batch_columns, lsm_call_request

    lib = _abi.load()
    c = _workloads.ragged_columns(args.ragged_contracts, seed=41)
    req = _workloads.ragged_request(c)
    nodes = sum(len(_workloads.ragged_row_as_call(c, r)["schedule_times"]) for r in range(c.rows))
    result = batch_columns(req.rows)
    err = _abi.FoError()
    g = _abi.FoRaggedGreeksColumns()
    arrays = {"delta": np.zeros(c.rows), "vega": np.zeros(c.rows), "d_l": np.zeros(nodes),
              "offsets": np.zeros(c.rows + 1, dtype=np.int64), "d_d": np.zeros(max(c.dividend_times.size, 1))}
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    g.delta, g.vega, g.log_discount_sensitivities = dp(arrays["delta"]), dp(arrays["vega"]), dp(arrays["d_l"])
    g.log_discount_capacity = nodes
    g.log_discount_offsets = arrays["offsets"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    g.dividend_sensitivities = dp(arrays["d_d"])
    steps = _workloads.ragged_path_steps(c)
    ms = (ctypes.c_double * 5)()
    launches = ctypes.c_uint64()
    out = {"workload": (f"ragged batch: {c.rows} contracts, paths per role log-uniform in [8192, 262144] "
                        f"(mean {float(c.paths.mean()):.0f}), 4-104 exercise dates, S0~U[20,500], K/S0~U[0.7,1.3], "
                        "sigma~U[0.05,0.8], T~U[0.1,3], r~U[0,0.08], even rows yield q~U[0,0.05], odd rows 1-6 cash "
                        "dividends, seed 41"),
           "contracts": c.rows, "path_steps_per_call": steps, "log_discount_sensitivities": nodes}
    calls = max(1, min(args.steps, 3))
    for name, greeks in (("plain", None), ("price_and_greeks", ctypes.byref(g))):
        def call() -> None:
            if lib.fo_price_lsm_ragged_f64(executor.raw, ctypes.byref(req.struct), ctypes.byref(result.struct), greeks,
                                           ctypes.byref(err)):
                raise RuntimeError(err.message.decode())
        call()
        kernel_ms = [0.0] * 5
        t0 = time.perf_counter()
        for _ in range(calls):
            call()
            lib.fo_executor_batch_kernel_ms(executor.raw, ms, 5, ctypes.byref(launches))
            kernel_ms = [a + b for a, b in zip(kernel_ms, ms, strict=True)]
        wall = time.perf_counter() - t0
        device_ms = kernel_ms[0] / calls
        out[name] = {"device_ms_per_call": device_ms, "device_contracts_per_s": c.rows / (device_ms / 1e3),
                     "device_path_steps_per_s": steps / (device_ms / 1e3),
                     "e2e_contracts_per_s": c.rows * calls / wall, "e2e_ms_per_call": wall / calls * 1e3,
                     "kernels_ms": batch_kernel_ms(kernel_ms, calls),
                     "gpu_launches_per_call": int(launches.value), "launch_shape": batch_launch(lib, executor)}
    out["greeks_overhead"] = out["price_and_greeks"]["device_ms_per_call"] / out["plain"]["device_ms_per_call"]
    out["executors_ms_per_call"] = {"price_and_greeks": executor_times(lib, executor, call)}  # the last call() defined
    # The north-star comparison: the same contracts (same populations, so the same price and SE)
    # priced one by one on the plain per-contract path, against the batched price + Greeks call.
    import finoptions as fo

    api_executor = fo.CudaExecutor(device=executor.device)
    calls = [public_call_arguments(_workloads.ragged_row_as_call(c, r), api_executor) for r in range(c.rows)]
    plain = one_by_one(calls, np.array(result.as_tuple()[0]), np.array(result.as_tuple()[2]))
    out["plain_per_contract"] = plain
    out["batched_vs_plain_same_contracts"] = {
        "batched": "fo_price_lsm_ragged_f64 with the adjoint Greeks, host columns in and out",
        "plain": plain["api"],
        "batched_contracts_per_s": out["price_and_greeks"]["e2e_contracts_per_s"],
        "plain_contracts_per_s": plain["contracts_per_s"],
        "ratio": out["price_and_greeks"]["e2e_contracts_per_s"] / plain["contracts_per_s"],
    }
    out["sample_greeks"] = {"delta_row0": float(arrays["delta"][0]), "vega_row0": float(arrays["vega"][0])}
    threads = cpu_threads()
    t0 = time.perf_counter()
    sample_steps = 0
    for r in range(RAGGED_SAMPLE):
        kw = _workloads.ragged_row_as_call(c, r)
        _oracle.price_lsm_call(lsm_call_request(**kw), threads)
        sample_steps += 2 * int(c.paths[r]) * (len(kw["schedule_times"]) - 1)
    cpu_s = time.perf_counter() - t0
    rate = sample_steps / cpu_s
    out["cpu_baseline"] = {"kind": "port", "cores": threads, "path_steps_per_s": rate,
                           "contracts_per_s": c.rows / (steps / rate),
                           "sample": f"the first {RAGGED_SAMPLE} contracts priced one by one ({cpu_s:.2f} s); the "
                                     "whole batch scaled by path-steps; Greeks by bump-and-reprice would multiply it "
                                     "by 2 x (2 + mesh nodes + cash events) + 1"}
    return out


# ---- price + adjoint Greeks ----------------------------------------------------------------------

GREEK_DIVIDENDS = ((13, 1.5), (39, 1.5))


def greeks_kwargs(paths: int = PATHS) -> dict:
    kw = workload_kwargs(paths)
    kw["dividend_nodes"] = [n for n, _ in GREEK_DIVIDENDS]
    kw["dividend_amounts"] = [a for _, a in GREEK_DIVIDENDS]
    return kw


def run_greeks(args: argparse.Namespace, executor) -> dict:
    """The weekly contract with cash dividends of 1.5 at weeks 13 and 39: device time per contract
    of the plain pricing pass and of the pass that also forms delta, vega, 53 log-discount and 2
    dividend sensitivities (same evaluation, same standard error)."""
    from finoptions import _abi
    from finoptions._requests import lsm_call_greeks, lsm_call_request, lsm_call_result

    lib = _abi.load()
    paths = args.paths
    kw = greeks_kwargs(paths)
    req = lsm_call_request(**kw)
    err = _abi.FoError()
    elapsed = ctypes.c_double()
    kernel_ms = (ctypes.c_double * 8)()
    steps = max(3, min(args.steps, 50))
    timings = {}
    for name, greeks in (("plain", 0), ("price_and_greeks", 1)):
        plan = ctypes.c_void_p()
        if lib.fo_lsm_call_plan_create(executor.raw, ctypes.byref(req.struct), ctypes.byref(plan), ctypes.byref(err)):
            raise RuntimeError(err.message.decode())
        lib.fo_lsm_call_plan_set_greeks(plan, greeks, ctypes.byref(err))
        lib.fo_lsm_call_plan_time_launches(plan, args.warmup, ctypes.byref(elapsed), None, 0, ctypes.byref(err))
        if lib.fo_lsm_call_plan_time_launches(plan, steps, ctypes.byref(elapsed), kernel_ms, 8, ctypes.byref(err)):
            raise RuntimeError(err.message.decode())
        res = lsm_call_result(req.exercise_rows)
        if lib.fo_lsm_call_plan_collect(plan, ctypes.byref(res.struct), ctypes.byref(err)):
            raise RuntimeError(err.message.decode())
        entry = {"ms_per_contract": elapsed.value / steps, "evaluate_ms": kernel_ms[3] / steps,
                 "price": res.as_tuple()[0], "standard_error": res.as_tuple()[3]}
        if greeks:
            g, d_l, d_d = lsm_call_greeks(STEPS_IN_GRID + 1, len(GREEK_DIVIDENDS))
            lib.fo_lsm_call_plan_greeks(plan, ctypes.byref(g), ctypes.byref(err))
            entry.update(delta=g.delta, vega=g.vega, dividend_sensitivities=d_d.tolist(),
                         log_discount_sensitivity_sum=float(d_l.sum()))
        lib.fo_lsm_call_plan_destroy(plan)
        timings[name] = entry
    sensitivities = 2 + (STEPS_IN_GRID + 1) + len(GREEK_DIVIDENDS)
    reprices = 2 * (2 + STEPS_IN_GRID + len(GREEK_DIVIDENDS))  # central bumps; L_0 is pinned at 0
    threads = cpu_threads()
    t0 = time.perf_counter()
    oracle_price(greeks_kwargs(paths), threads)
    cpu_price_s = time.perf_counter() - t0
    plain_ms, greeks_ms = timings["plain"]["ms_per_contract"], timings["price_and_greeks"]["ms_per_contract"]
    return {
        "workload": "weekly contract of the headline with cash dividends 1.5 at weeks 13 and 39 (liquidator)",
        "paths": paths,
        "sensitivities": sensitivities,
        "plain": timings["plain"],
        "price_and_greeks": timings["price_and_greeks"],
        "greeks_overhead": greeks_ms / plain_ms,
        "contracts_per_s": {"plain": 1e3 / plain_ms, "price_and_greeks": 1e3 / greeks_ms},
        "bump_and_reprice_gpu_ms": reprices * plain_ms,
        "cpu_baseline": {"kind": "port", "cores": threads, "one_price_s": cpu_price_s,
                         "bump_and_reprice_s": (1 + reprices) * cpu_price_s,
                         "sample": f"one oracle price of this contract timed; {reprices} more for central bumps"},
    }


# ---- batched grouped workload ------------------------------------------------------------------

GROUPED_STATES = 4096
GROUPED_STRIKES = 8
GROUPED_PATHS = 32768
GROUPED_SAMPLE_STATES = 48
GROUPED_PLAIN_SAMPLE = 1024


def grouped_algorithmic_bytes(c, paths: int) -> dict:
    """Algorithmic HBM bytes per call: the training rows are written once by the simulation; each
    (state, strike) problem reads its state's rows once and reads + writes its values per row."""
    import numpy as np

    rows = np.diff(c.exercise_offsets) + 1  # explicit exercise dates + expiry (origin excluded)
    strikes = np.diff(c.group_offsets.astype(np.int64))
    return {
        "batch_simulate_kernel": int((8 * rows * paths).sum()),
        "batch_backward_kernel": int((strikes * (8 * rows * paths + 16 * (rows - 1) * paths)).sum()),
    }


def fit_traffic(kernel: str, algorithmic: dict) -> int | None:
    """DRAM bytes of the batch fit kernel per call: the committed ncu capture's DRAM bytes per
    algorithmic byte (profiles/traffic.json, taken at 128 states) times this call's algorithmic
    bytes, since both grow with the states priced."""
    path = ROOT / "profiles" / "traffic.json"
    if kernel != "batch_fit_kernel" or not path.is_file():
        return None
    entry = json.loads(path.read_text()).get("batch_fit_kernel")
    if entry is None:
        return None
    return int(float(entry["dram_bytes_per_algorithmic_byte"]) * algorithmic["batch_backward_kernel"])


def batch_kernel_ms(kernel_ms: list, calls: int) -> dict:
    """Per-call device milliseconds of a batch call's graph, split into the phase kernels when the
    executor ran them (fo_executor_batch_kernel_ms slots 1..3)."""
    out = {"graph": round(kernel_ms[0] / calls, 3)}
    if any(kernel_ms[1:4]):
        out.update(simulate=round(kernel_ms[1] / calls, 3), fit=round(kernel_ms[2] / calls, 3),
                   evaluate=round(kernel_ms[3] / calls, 3))
    return out


def executor_times(lib, executor, call, repeats: int = 2) -> dict:
    """Device milliseconds per call of the batch under each executor, with the autotuner's other
    choices kept (the persistent launch at as many CTAs per SM as fit); the autotuner is restored
    afterwards. The results are the same bit for bit under both."""
    from finoptions import _abi

    info = _abi.FoBatchLaunchInfo()
    lib.fo_executor_batch_launch(executor.raw, ctypes.byref(info))
    chosen = info.tuning
    ms = (ctypes.c_double * 5)()
    n = ctypes.c_uint64()
    err = _abi.FoError()
    out = {}
    try:
        for phases, name in ((0, "one_persistent_launch"), (1, "phase_kernels")):
            shape = _abi.FoBatchTuning(chosen.sim_blocks, chosen.eval_blocks, chosen.strikes, 0, phases)
            if lib.fo_executor_set_batch_tuning(executor.raw, 0, ctypes.byref(shape), ctypes.byref(err)):
                raise RuntimeError(err.message.decode())
            call()  # captures the graph of this shape
            total = 0.0
            for _ in range(repeats):
                call()
                lib.fo_executor_batch_kernel_ms(executor.raw, ms, 5, ctypes.byref(n))
                total += ms[0]
            out[name] = round(total / repeats, 2)
    finally:
        lib.fo_executor_set_batch_tuning(executor.raw, 1, None, ctypes.byref(err))
    return out


def batch_launch(lib, executor) -> dict:
    """The launch shape the executor used for its last batch call (autotuned per shape class)."""
    from finoptions import _abi

    info = _abi.FoBatchLaunchInfo()
    lib.fo_executor_batch_launch(executor.raw, ctypes.byref(info))
    t = info.tuning
    return {"sim_blocks_per_item": t.sim_blocks, "eval_blocks_per_item": t.eval_blocks,
            "strikes_per_eval_item": t.strikes, "ctas_per_sm": t.ctas_per_sm or "max", "ctas": info.grid,
            "work_items": int(info.items), "chosen_by": ("caller", "autotuner (cached)", "autotuner")[info.source],
            "executor": "phase kernels (simulation, fit, evaluation, summary)" if t.phases else "one persistent launch",
            "graph_replays_last_call": int(info.graph_replays), "graph_captures_last_call": int(info.graph_captures)}


def run_grouped(args: argparse.Namespace, executor) -> dict:
    """The grouped batch (4096 states x 8 strikes, 32,768 + 32,768 paths per state) through the C
    ABI with host columns in and host result columns out, per call."""
    import _workloads
    from finoptions import _abi
    from finoptions._requests import batch_columns

    lib = _abi.load()
    states = args.batched_states
    cols = _workloads.grouped_columns(states, GROUPED_STRIKES, seed=23)
    req = _workloads.grouped_request(cols, GROUPED_PATHS)
    result = batch_columns(req.rows)
    err = _abi.FoError()

    def call() -> None:
        st = lib.fo_price_lsm_grouped_f64(executor.raw, ctypes.byref(req.struct), ctypes.byref(result.struct),
                                          ctypes.byref(err))
        if st:
            raise RuntimeError(err.message.decode())

    steps = max(1, min(args.steps, 5))
    for _ in range(2):
        call()
    clocks = ClockSampler(executor.device)
    kernel_ms = [0.0] * 5
    launches = 0
    ms = (ctypes.c_double * 5)()
    n_launch = ctypes.c_uint64()
    with clocks:
        t0 = time.perf_counter()
        for _ in range(steps):
            call()
            lib.fo_executor_batch_kernel_ms(executor.raw, ms, 5, ctypes.byref(n_launch))
            kernel_ms = [a + b for a, b in zip(kernel_ms, ms, strict=True)]
            launches += int(n_launch.value)
        wall = time.perf_counter() - t0
    h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
    lib.fo_executor_batch_transfer_bytes(executor.raw, ctypes.byref(h2d), ctypes.byref(d2h))
    device_ms = kernel_ms[0] / steps
    contracts = req.rows
    steps_per_call = _workloads.path_steps(cols, GROUPED_PATHS)
    algorithmic = grouped_algorithmic_bytes(cols, GROUPED_PATHS)
    hbm_peak, peak_kind = measured_peaks()
    # One persistent launch per call: its algorithmic bytes are the training rows' store and the
    # fits' reads and value round trips; its time also holds the (issue-bound) evaluation.
    launch_bytes = sum(algorithmic.values())
    kernels = {"batch_persistent_kernel": {"ms_per_call": round(device_ms, 4), "share": 1.0,
                                           "algorithmic_bytes": launch_bytes,
                                           "achieved_gbs": round(launch_bytes / (device_ms / 1e3) / 1e9, 1)}}
    shape = batch_launch(lib, executor)
    executors = executor_times(lib, executor, call)
    dominant = "batch_persistent_kernel"
    achieved = launch_bytes / (device_ms / 1e3) / 1e9
    bound = "hbm (fits) + issue (simulation, evaluation)"
    phases = batch_kernel_ms(kernel_ms, steps)
    if len(phases) > 1:  # the phase executor: one kernel per item kind, inside the same graph
        kernels = {"batch_" + name + "_kernel": {"ms_per_call": ms, "share": round(ms / device_ms, 4)}
                   for name, ms in phases.items() if name != "graph"}
        for name, key in (("simulate", "batch_simulate_kernel"), ("fit", "batch_backward_kernel")):
            k = kernels["batch_" + name + "_kernel"]
            k.update(algorithmic_bytes=algorithmic[key],
                     achieved_gbs=round(algorithmic[key] / (k["ms_per_call"] / 1e3) / 1e9, 1))
        dominant = "batch_fit_kernel"
        achieved = kernels[dominant]["achieved_gbs"]
        bound = "latency (one CTA per problem, row by row; values and spots from L2 / HBM)"

    # The same contracts one by one on the plain per-contract path: the first GROUPED_PLAIN_SAMPLE
    # rows (whole states), each repricing its state's populations (same price and SE as the batch).
    import finoptions as fo
    import numpy as np

    api_executor = fo.CudaExecutor(device=executor.device)
    sample_rows = min(contracts, GROUPED_PLAIN_SAMPLE)
    calls = [public_call_arguments(_workloads.grouped_row_as_call(cols, r, GROUPED_PATHS), api_executor)
             for r in range(sample_rows)]
    plain = one_by_one(calls, np.array(result.as_tuple()[0][:sample_rows]), np.array(result.as_tuple()[2][:sample_rows]))
    plain["sample"] = f"the first {sample_rows} of the {contracts} contracts ({sample_rows // GROUPED_STRIKES} states)"
    e2e_contracts_per_s = contracts * steps / wall
    # CPU restatement of the reference's group-parallel CpuExecutor on a bounded sample of states.
    threads = cpu_threads()
    sample = _workloads.grouped_columns(GROUPED_SAMPLE_STATES, GROUPED_STRIKES, seed=23)
    sample_req = _workloads.grouped_request(sample, GROUPED_PATHS)
    import _oracle

    t0 = time.perf_counter()
    _oracle.price_lsm_grouped(sample_req, threads)
    cpu_s = time.perf_counter() - t0
    return {
        "workload": (f"grouped batch: {states} states x {GROUPED_STRIKES} strikes (K/S0 0.8..1.2), "
                     f"{GROUPED_PATHS} + {GROUPED_PATHS} paths per state, explicit meshes of 12-52 dates, "
                     "0-4 exercise-aligned cash dividends (liquidator), insufficient support = continue, seed 23"),
        "contracts": contracts,
        "path_steps_per_call": steps_per_call,
        "calls": steps,
        "device_ms_per_call": device_ms,
        "device_contracts_per_s": contracts / (device_ms / 1e3),
        "device_path_steps_per_s": steps_per_call / (device_ms / 1e3),
        "e2e": {"contracts_per_s": contracts * steps / wall, "path_steps_per_s": steps_per_call * steps / wall,
                "ms_per_call": wall / steps * 1e3, "h2d_bytes_per_step": int(h2d.value),
                "d2h_bytes_per_step": int(d2h.value), "api": "fo_price_lsm_grouped_f64 (host columns in and out)"},
        "gpu_launches": launches,
        "launch_shape": shape,
        "executors_ms_per_call": executors,
        "kernels": kernels,
        "roofline": {"kernel": dominant, "bound": bound,
                     "achieved": round(achieved, 1), "peak": hbm_peak, "peak_source": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": fit_traffic(dominant, algorithmic)},
        "clocks": clocks.report(),
        "plain_per_contract": plain,
        "batched_vs_plain_same_contracts": {
            "batched": "fo_price_lsm_grouped_f64, host columns in and out", "plain": plain["api"],
            "batched_contracts_per_s": e2e_contracts_per_s, "plain_contracts_per_s": plain["contracts_per_s"],
            "ratio": e2e_contracts_per_s / plain["contracts_per_s"]},
        "cpu_baseline": {"contracts_per_s": GROUPED_SAMPLE_STATES * GROUPED_STRIKES / cpu_s,
                         "path_steps_per_s": _workloads.path_steps(sample, GROUPED_PATHS) / cpu_s, "cores": threads,
                         "kind": "port", "sample": f"the first {GROUPED_SAMPLE_STATES} states of the workload "
                                                   f"({cpu_s:.2f} s on {threads} threads)"},
    }


def cpu_baseline(paths: int = PATHS) -> dict:
    """The CPU restatement of the reference engine (path-parallel simulation on every host thread,
    serial fit and evaluation per contract) on one full contract of the workload."""
    threads = cpu_threads()
    kwargs = workload_kwargs(paths)
    oracle_price(workload_kwargs(1 << 14), threads)  # load + warm
    t0 = time.perf_counter()
    oracle_price(kwargs, threads)
    seconds = time.perf_counter() - t0
    return {"value": path_steps(paths) / seconds, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one full contract of the workload ({seconds:.2f} s on {threads} threads)"}


# ---- reference arm -----------------------------------------------------------------------------


def run_reference(args: argparse.Namespace) -> dict | None:
    """The reference's CpuExecutor path (its CPU restatement; the Rust reference cannot be built
    here) on every host thread: each step prices the full workload contract, 2^20 + 2^20 paths,
    the configuration the line names."""
    rank, world, _ = dist_info()
    if rank != 0:
        return None
    threads = cpu_threads()
    paths = args.paths
    kwargs = workload_kwargs(paths)
    for _ in range(args.warmup):
        oracle_price(kwargs, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle_price(kwargs, threads)
    seconds = time.perf_counter() - t0
    value = path_steps(paths) * args.steps / seconds
    sample = (f"each step prices the whole workload contract ({paths} + {paths} paths) on {threads} host threads "
              "with the CPU restatement of the reference engine (path-parallel simulation, serial fit and evaluation)")
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": seconds / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(paths),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=None,
                        help="timed steps (default 200; 10 for --impl reference, whose steps take seconds each)")
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--paths", type=int, default=PATHS, help="paths per role (profiling captures shrink it)")
    parser.add_argument("--skip-batched", action="store_true", help="omit the grouped-batch section")
    parser.add_argument("--skip-greeks", action="store_true", help="omit the price + Greeks section")
    parser.add_argument("--skip-ragged", action="store_true", help="omit the ragged-batch section")
    parser.add_argument("--ragged-contracts", type=int, default=RAGGED_CONTRACTS,
                        help="contracts of the ragged-batch section (profiling captures shrink it)")
    parser.add_argument("--batched-states", type=int, default=GROUPED_STATES,
                        help="states of the grouped-batch section (profiling captures shrink it)")
    args = parser.parse_args()
    if args.paths < 2:
        parser.error("--paths must be at least 2")
    if args.steps is None:
        args.steps = 10 if args.impl == "reference" else 200
    if args.warmup < 3:
        args.warmup = 3
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
