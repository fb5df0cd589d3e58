"""Typed exceptions with the reference's hierarchy (crates/finoptions-python/src/lib.rs:57-64)."""

from __future__ import annotations


class InputError(ValueError):
    """Invalid request, financial input, or validation failure."""


class BatchError(ValueError):
    """Malformed ragged (Arrow-style) batch structure."""


class ExecutionError(RuntimeError):
    """Executor construction or device failure."""


class SimulationError(RuntimeError):
    """Path-simulation failure."""


class LsmError(RuntimeError):
    """Simulation, regression, support, or fixed-policy evaluation failure inside LSM."""


_BY_KIND = {1: InputError, 2: LsmError, 3: SimulationError, 4: ExecutionError, 5: BatchError}


def raise_for(status: int, error: object) -> None:
    """Raise the typed exception for a non-zero fo_status with the native message."""
    if status == 0:
        return
    kind = getattr(error, "kind", status) or status
    message = getattr(error, "message", b"")
    text = message.decode("utf-8", "replace") if isinstance(message, bytes) else str(message)
    exc = _BY_KIND.get(int(kind), ExecutionError)(text)
    exc.code = int(getattr(error, "code", 0))  # type: ignore[attr-defined]
    exc.row = int(getattr(error, "row", -1))  # type: ignore[attr-defined]
    exc.group = int(getattr(error, "group", -1))  # type: ignore[attr-defined]
    exc.node = int(getattr(error, "node", -1))  # type: ignore[attr-defined]
    exc.path = int(getattr(error, "path", -1))  # type: ignore[attr-defined]
    raise exc
