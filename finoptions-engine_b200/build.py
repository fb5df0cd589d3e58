"""Build the B200 engine's shared library in-tree for sm_100a.

    python finoptions-engine_b200/build.py [--verbose]

Produces finoptions-engine_b200/finoptions/_lib/libfinoptions_cuda.so from csrc/. Every kernel is
compiled for sm_100a only; --fmad=false keeps multiply-adds unfused except where the source calls
fma(), matching the reference's explicit mul_add usage.
"""

from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "finoptions" / "_lib"
OUT = OUT_DIR / "libfinoptions_cuda.so"
BUILD_DIR = HERE / "_build"
SOURCES = ("host.cpp", "capi.cu", "lsm_kernels.cu", "lsm_greeks.cu", "lsm_persistent.cu", "lsm_grouped.cu")
NVCC_FLAGS = (
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math", "-Xcompiler", "-ffp-contract=off",
    "-DFO_PACKAGE_VERSION=\"0.1.0\"",
)


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        msg = "nvcc not found; the B200 engine cannot be built"
        raise RuntimeError(msg)
    return path


def _digest() -> str:
    h = hashlib.sha256()
    for f in sorted(CSRC.glob("*")):
        if f.suffix in {".cu", ".cuh", ".h", ".cpp"}:
            h.update(f.name.encode())
            h.update(f.read_bytes())
    h.update((HERE.parent / "include" / "finoptions_cuda.h").read_bytes())
    h.update(" ".join(NVCC_FLAGS).encode())
    return h.hexdigest()


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every source for sm_100a and link the shared library; skip when up to date."""
    stamp = OUT_DIR / ".build_digest"
    digest = _digest()
    if not force and OUT.is_file() and stamp.is_file() and stamp.read_text() == digest:
        return OUT
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    def compile_one(src: str) -> tuple[str, subprocess.CompletedProcess]:
        obj = BUILD_DIR / (Path(src).stem + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-x", "cu", "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        return str(obj), subprocess.run(cmd, capture_output=True, text=True, check=False)

    # The translation units are independent: compile them side by side.
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as pool:
        compiled = list(pool.map(compile_one, SOURCES))
    objects = []
    for src, (obj, result) in zip(SOURCES, compiled, strict=True):
        if verbose or result.returncode:
            sys.stderr.write(result.stdout + result.stderr)
        if result.returncode:
            msg = f"nvcc failed for {src}"
            raise RuntimeError(msg)
        objects.append(obj)
    tmp = OUT.with_suffix(".so.tmp")
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp), *objects,
            "-Xcompiler", "-fPIC"]
    result = subprocess.run(link, capture_output=True, text=True, check=False)
    if result.returncode:
        sys.stderr.write(result.stdout + result.stderr)
        msg = "linking libfinoptions_cuda.so failed"
        raise RuntimeError(msg)
    os.replace(tmp, OUT)
    stamp.write_text(digest)
    return OUT


if __name__ == "__main__":
    parser = argparse.ArgumentParser()
    parser.add_argument("--verbose", action="store_true")
    parser.add_argument("--force", action="store_true")
    args = parser.parse_args()
    print(build(verbose=args.verbose, force=args.force))
