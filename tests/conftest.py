"""Test configuration: the `gpu` marker, import paths and the in-tree engine build."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PACKAGE_DIR = ROOT / "finoptions-engine_b200"
for path in (PACKAGE_DIR, ROOT / "tests"):
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) device")


def _ensure_library() -> None:
    sys.path.insert(0, str(PACKAGE_DIR))
    import build  # noqa: PLC0415 - the package's build script

    build.build()


_ensure_library()


@pytest.fixture(scope="session")
def executor():
    """One CudaExecutor for the GPU tests (fails loudly without a device)."""
    import finoptions  # noqa: PLC0415

    return finoptions.CudaExecutor(device=0)


@pytest.fixture(scope="session")
def native_executor(executor):
    """The native handle of the session executor."""
    from finoptions.simulation import native_executor as handle  # noqa: PLC0415

    return handle(executor)
