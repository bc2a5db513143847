"""Error hierarchy with the reference's class names (ertm/exceptions.py:12-64).

Callers that catch ``SolverError`` / ``ImagingError`` around the reference
keep working: the GPU path raises the same classes for the same triggers.
"""

from __future__ import annotations

from typing import Any


class ERTMError(Exception):
    """Base of every expected failure; carries an optional context dict."""

    def __init__(self, message: str, *, context: dict[str, Any] | None = None) -> None:
        self.message = str(message)
        self.context = dict(context or {})
        super().__init__(self.message)

    def __str__(self) -> str:
        if not self.context:
            return self.message
        return f"{self.message} (" + ", ".join(f"{k}={v!r}" for k, v in self.context.items()) + ")"

    def to_dict(self) -> dict[str, Any]:
        return {"type": type(self).__name__, "message": self.message, "context": self.context}


class ConfigError(ERTMError):
    """Invalid configuration value."""


class ModelError(ERTMError):
    """Invalid earth model."""


class SolverError(ERTMError):
    """Propagation input or runtime failure (CFL, components, receivers, device)."""


class ImagingError(ERTMError):
    """Imaging input or condition failure."""


class NonFiniteWavefieldError(SolverError):
    """A wavefield became NaN or infinite during a run (an unstable or
    overflowing propagation), detected on the device by the stress phase.
    No counterpart in the reference, which finishes such a run with a
    non-finite image."""


class DataError(ERTMError):
    """Data format failure."""


class PipelineError(ERTMError):
    """Orchestration failure."""
