"""The engine's corrected division (fo_core.cuh `divide`) against IEEE binary64 division on the B200.

The kernels divide the in-the-money spot by the strike and the centred predictor by the fitted
scale with a reciprocal and Markstein's correction step; the result must be the correctly rounded
quotient, i.e. bit-identical to `a / b`, on the operand ranges the engine meets.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
BUILD = HERE / "native" / "_build"


def harness() -> ctypes.CDLL:
    lib = BUILD / "libdivide_harness.so"
    src = HERE / "native" / "divide_harness.cu"
    if not lib.is_file() or lib.stat().st_mtime < max(src.stat().st_mtime,
                                                      (HERE.parent / "finoptions-engine_b200/csrc/fo_core.cuh").stat().st_mtime):
        BUILD.mkdir(parents=True, exist_ok=True)
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-std=c++17",
                        "-shared", "-Xcompiler", "-fPIC", str(src), "-o", str(lib)], check=True)
    dll = ctypes.CDLL(str(lib))
    dll.divide_check.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong),
                                 ctypes.POINTER(ctypes.c_double)]
    dll.divide_check.restype = ctypes.c_int
    return dll


@pytest.mark.parametrize("family", [0, 1, 2, 3], ids=["spot_over_strike", "predictor_over_scale",
                                                      "all_ones_divisor", "near_powers_of_two"])
def test_corrected_division_is_correctly_rounded(family: int) -> None:
    count = ctypes.c_ulonglong()
    first = (ctypes.c_double * 2)()
    assert harness().divide_check(1 << 24, family, ctypes.byref(count), first) == 0
    assert count.value == 0, f"{count.value} mismatches; first {first[0]!r} / {first[1]!r}"
