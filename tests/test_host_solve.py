"""The device regression solve, compiled for the host, against the oracle's sequential
Stieltjes fit (regression.rs:369-523) on in-the-money populations of realistic shape."""

from __future__ import annotations

import ctypes
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import _oracle

HERE = Path(__file__).resolve().parent
BUILD = HERE / "native" / "_build"


@pytest.fixture(scope="module")
def harness() -> ctypes.CDLL:
    BUILD.mkdir(parents=True, exist_ok=True)
    lib = BUILD / "libsolve_harness.so"
    src = HERE / "native" / "solve_harness.cpp"
    if not lib.is_file() or lib.stat().st_mtime < max(src.stat().st_mtime, (HERE.parent / "finoptions-engine_b200" / "csrc" / "fo_core.cuh").stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", str(src), "-o", str(lib)],
                       check=True)
    h = ctypes.CDLL(str(lib))
    h.harness_fit.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, ctypes.c_int,
                              ctypes.c_int, ctypes.c_void_p]
    return h


def population(rng: np.random.Generator, n: int, sigma: float, moneyness: float) -> tuple[np.ndarray, np.ndarray]:
    s = 100.0 * np.exp(sigma * rng.standard_normal(4 * n))
    k = 100.0 * moneyness
    s = s[s > k][:n]
    y = np.maximum(s * np.exp(0.3 * sigma * rng.standard_normal(s.size)) - k, 0.0) * 0.99
    return s / k, y


@pytest.mark.parametrize("degree", [0, 1, 2, 3, 4])
def test_one_pass_moment_solve_matches_the_sequential_reference_fit(harness, degree) -> None:
    rng = np.random.default_rng(17 + degree)
    worst = 0.0
    for trial in range(24):
        n = 40 + trial * 7 if trial % 3 == 0 else 20000
        x, y = population(rng, n, 0.05 + 0.07 * (trial % 7), 0.7 + 0.1 * (trial % 5))
        code, model, _ = _oracle.fit_regression(x, y, degree)
        if code != 0:
            continue
        for offset in (-1.5, -0.3, 0.0, 0.4, 1.5):  # pivot distance from the mean, in scales
            pivot = (1.2 if degree == 0 else model[0]) + offset * model[1]
            ours = np.zeros(22)
            status = harness.harness_fit(x.ctypes.data, y.ctypes.data, x.size, pivot, degree, 4, ours.ctypes.data)
            assert status // 10 == 0 and status % 10 == 0, status
            assert ours[20] == model[20]  # rank
            assert abs(ours[21] - model[21]) <= 1e-8 * model[21]
            if degree:
                assert abs(ours[0] - model[0]) <= 1e-13 * abs(model[0])
                assert abs(ours[1] - model[1]) <= 1e-12 * model[1]
            reference = _oracle.predict(model, degree, x)
            predicted = _oracle.predict(ours, degree, x)
            worst = max(worst, float(np.max(np.abs(predicted - reference)) / np.max(np.abs(reference))))
    assert worst <= 1e-12


def test_rank_limit_is_the_last_spread_the_rank_test_accepts(harness) -> None:
    """norm / n <= rank_limit(tol) is the solve's rank test sqrt(norm / n) <= tol (correctly
    rounded square root), so the warp solve needs no square root per step."""
    harness.harness_rank_limit.argtypes = [ctypes.c_double]
    harness.harness_rank_limit.restype = ctypes.c_double
    rng = np.random.default_rng(5)
    tolerances = [1e-12, 1e-8, 0.5, 0.3, math.nextafter(1.0, 0.0), 1e-300, 5e-324, *10.0 ** rng.uniform(-16, -0.01, 2000)]
    for tol in tolerances:
        q = harness.harness_rank_limit(float(tol))
        assert q >= 0.0 and math.sqrt(q) <= tol, tol
        assert math.sqrt(math.nextafter(q, math.inf)) > tol, tol


@pytest.mark.parametrize("degree", [0, 1, 2, 3, 4])
def test_per_degree_predictor_is_bit_identical_to_the_runtime_degree_predictor(harness, degree) -> None:
    """The kernels that apply a fitted policy path by path are instantiated per degree
    (predict_continuation_d<D>); each instance must predict exactly what the runtime-degree
    predictor does, failures (non-finite predictor or prediction) included."""
    harness.harness_predict_mismatches.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64]
    rng = np.random.default_rng(71 + degree)
    for trial in range(20):
        model = np.concatenate([[rng.uniform(0.8, 1.6), rng.uniform(0.02, 0.4)], rng.normal(0, 1.5, 4),
                                rng.uniform(0.1, 2.0, 4), rng.normal(0, 5.0, 5)])
        x = rng.uniform(0.5, 3.0, 4000)
        x[:4] = [math.inf, -math.inf, math.nan, 1e308]
        if trial == 0:
            model[10] = math.inf  # non-finite prediction
        assert harness.harness_predict_mismatches(model.ctypes.data, degree, x.ctypes.data, x.size) == 0
