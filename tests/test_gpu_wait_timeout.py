"""The backward kernel's grid wait gives up instead of hanging.

The persistent backward kernel synchronises its CTAs through an arrival counter. If a CTA never
arrives, every waiting warp gives up after its time limit, raises the status word's timeout flag
(reported by the host as FO_CODE_BARRIER_TIMEOUT) and returns, and the context stays usable. The
failure is made on purpose here without any fault: the waits watch a counter that nothing
increments.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
BUILD = HERE / "native" / "_build"
CSRC = HERE.parent / "finoptions-engine_b200" / "csrc"
BLOCKS = 4


def harness() -> ctypes.CDLL:
    lib = BUILD / "libwait_harness.so"
    src = HERE / "native" / "wait_harness.cu"
    deps = [src, CSRC / "lsm_sync.cuh", CSRC / "lsm_device.cuh", CSRC / "fo_core.cuh"]
    if not lib.is_file() or lib.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        BUILD.mkdir(parents=True, exist_ok=True)
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-std=c++17",
                        "-shared", "-Xcompiler", "-fPIC", str(src), "-o", str(lib)], check=True)
    dll = ctypes.CDLL(str(lib))
    dll.wait_check.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_ulonglong, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_ulonglong),
                               ctypes.POINTER(ctypes.c_uint)]
    dll.wait_check.restype = ctypes.c_int
    return dll


def run(arrivals: int, target: int, limit_ns: int) -> tuple[list[int], list[int], int]:
    passed = (ctypes.c_int * BLOCKS)()
    elapsed = (ctypes.c_ulonglong * BLOCKS)()
    flag = ctypes.c_uint()
    assert harness().wait_check(arrivals, target, limit_ns, BLOCKS, passed, elapsed, ctypes.byref(flag)) == 0
    return list(passed), list(elapsed), flag.value


def test_a_wait_that_nobody_releases_times_out_and_the_context_stays_usable() -> None:
    limit = 500_000_000  # 0.5 s
    passed, elapsed, flag = run(arrivals=0, target=1, limit_ns=limit)
    assert passed == [0] * BLOCKS and flag == 1
    # The first warp to give up raises the flag; the others leave at their next check.
    # (a block that started later may leave on the flag slightly before its own limit)
    assert min(elapsed) >= 0.9 * limit and max(elapsed) < limit + 1_000_000_000
    # Same device, next launch: a wait whose arrivals are complete passes at once.
    passed, elapsed, flag = run(arrivals=2 * BLOCKS, target=2 * BLOCKS, limit_ns=limit)
    assert passed == [1] * BLOCKS and flag == 0
    assert max(elapsed) < limit
