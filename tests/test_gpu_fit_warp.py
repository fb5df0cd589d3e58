"""The backward kernel's warp-wide regression solve is bit-identical to the one-thread solve.

fit_continuation_warp spreads fit_near_pivot's binomial shift and Stieltjes recurrence over the
lanes of a warp with every value computed by the same binary64 operations in the same order, so
the two fitted models must agree byte for byte: on realistic in-the-money populations at pivots
on both sides of the mean (near pivots take the warp path, far ones the double-double fallback),
and on every failure the solve reports (degenerate predictor, rank deficiency at each step,
non-finite sums).
"""

from __future__ import annotations

import ctypes
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
BUILD = HERE / "native" / "_build"
CSRC = HERE.parent / "finoptions-engine_b200" / "csrc"
POWER_SUMS, SLOTS = 9, 14
STATUS_OFFSET = 168  # FitModel: mean, scale, inv_scale, alpha[4], beta[4], coef[5], norm[5], status


class FitCase(ctypes.Structure):
    _fields_ = [("sums", ctypes.c_double * (2 * SLOTS)), ("pivot", ctypes.c_double), ("count", ctypes.c_uint64),
                ("degree", ctypes.c_int), ("rank_tolerance", ctypes.c_double), ("rank_limit", ctypes.c_double)]


@pytest.fixture(scope="module")
def harness() -> ctypes.CDLL:
    lib = BUILD / "libfit_harness.so"
    src = HERE / "native" / "fit_harness.cu"
    deps = [src, CSRC / "lsm_fit_warp.cuh", CSRC / "fo_core.cuh"]
    if not lib.is_file() or lib.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        BUILD.mkdir(parents=True, exist_ok=True)
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-std=c++17",
                        "-shared", "-Xcompiler", "-fPIC", str(src), "-o", str(lib)], check=True)
    dll = ctypes.CDLL(str(lib))
    dll.fit_compare.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    assert dll.fit_case_bytes() == ctypes.sizeof(FitCase)
    return dll


def dd_sum(terms: np.ndarray) -> tuple[float, float]:
    hi = math.fsum(terms.tolist())
    return hi, math.fsum([*terms.tolist(), -hi])


def case(x: np.ndarray, y: np.ndarray, pivot: float, degree: int, tolerance: float = 1e-12) -> FitCase:
    d = x - pivot
    q = FitCase(pivot=pivot, count=x.size, degree=degree, rank_tolerance=tolerance)
    powers = np.ones_like(d)
    for k in range(POWER_SUMS):
        q.sums[2 * k], q.sums[2 * k + 1] = dd_sum(powers)
        if k <= 4:
            q.sums[2 * (POWER_SUMS + k)], q.sums[2 * (POWER_SUMS + k) + 1] = dd_sum(y * powers)
        powers = powers * d
    return q


def population(rng: np.random.Generator, n: int, sigma: float, moneyness: float) -> tuple[np.ndarray, np.ndarray]:
    s = 100.0 * np.exp(sigma * rng.standard_normal(4 * n))
    s = s[s > 100.0 * moneyness][:n]
    y = np.maximum(s * np.exp(0.3 * sigma * rng.standard_normal(s.size)) - 100.0 * moneyness, 0.0) * 0.99
    return s / (100.0 * moneyness), y


def cases() -> list[FitCase]:
    rng = np.random.default_rng(2024)
    out = []
    for degree in range(5):
        for trial in range(10):
            n = 30 + 11 * trial if trial % 2 else 5000
            x, y = population(rng, n, 0.04 + 0.06 * (trial % 5), 0.8 + 0.08 * (trial % 4))
            mean, sd = float(x.mean()), float(x.std())
            for offset in (-1.5, -0.6, -0.3, 0.0, 0.2, 0.4, 0.9, 1.5):
                out.append(case(x, y, mean + offset * sd, degree))
        # failures: two distinct predictors (rank deficient above degree 1), one repeated predictor
        # (degenerate scale), an aggressive rank tolerance, non-finite sums, the minimum population
        x2 = np.where(rng.random(60) < 0.5, 1.1, 1.3)
        out.append(case(x2, x2 * 2.0, 1.2, degree))
        out.append(case(np.full(40, 1.25), np.linspace(0.0, 1.0, 40), 1.2, degree))
        x, y = population(rng, 400, 0.1, 0.9)
        for tolerance in (0.02, 0.3, 0.9, 1.0):  # 1.0 fails at step 0 (norm / n of p_0 is 1)
            out.append(case(x, y, float(x.mean()), degree, tolerance=tolerance))
        for slot, value in ((POWER_SUMS + min(degree, 2), math.nan), (min(2 * degree, 8), math.inf),
                            (POWER_SUMS, math.inf)):
            q = case(x, y, float(x.mean()), degree)
            q.sums[2 * slot], q.sums[2 * slot + 1] = value, 0.0
            out.append(q)
        x, y = population(rng, degree + 1, 0.2, 0.9)
        out.append(case(x, y, float(x.mean()), degree))
        out.append(case(x, np.zeros_like(y), float(x.mean()), degree))
    return out


def test_warp_solve_is_bit_identical_to_the_one_thread_solve(harness) -> None:
    batch = cases()
    n = len(batch)
    array = (FitCase * n)(*batch)
    size = harness.fit_model_bytes()
    one = ctypes.create_string_buffer(size * n)
    warp = ctypes.create_string_buffer(size * n)
    assert harness.fit_compare(ctypes.addressof(array), n, one, warp) == 0
    statuses = set()
    for i in range(n):
        a, b = one.raw[i * size:(i + 1) * size], warp.raw[i * size:(i + 1) * size]
        assert a == b, f"case {i} (degree {batch[i].degree}) differs"
        statuses.add(int.from_bytes(a[STATUS_OFFSET:STATUS_OFFSET + 4], "little", signed=True))
    assert statuses == {0, 1, 2, 3}  # ok, degenerate predictor, rank deficient, non-finite
