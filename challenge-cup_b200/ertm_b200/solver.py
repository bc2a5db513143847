"""Forward-modelling facade with the reference interface (ertm/solver.py:34-154)."""

from __future__ import annotations

from typing import Any

import numpy as np

from .config import QConfig, SolverConfig
from .exceptions import SolverError
from .propagation import PropagationSpec, QOptions, check_stability, forward_shot, source_wavelet, stability_report
from .types import ShotRecord


class FiniteDifferenceSolver:
    name = "fd-two-way"

    def __init__(self, config: SolverConfig, q_config: QConfig | None = None) -> None:
        self.config = config
        self.config.validate()
        self.q_config = q_config or QConfig()

    def q_options(self, *, compensation: bool = False) -> QOptions | None:
        if self.config.engine != "viscoacoustic":
            return None
        q = self.q_config
        return QOptions(enabled=True, f_ref=float(q.f_ref), n_mechanisms=int(q.n_mechanisms),
                        band_ratio=float(q.band_ratio), compensation=bool(compensation), alpha_c=float(q.alpha_c),
                        amplitude_cap=float(q.amplitude_cap), lowpass_interval=int(q.lowpass_interval),
                        f_max=None if q.f_max is None else float(q.f_max), gain_budget_db=float(q.gain_budget_db))

    def spec(self, model: Any) -> PropagationSpec:
        """Uses the configured npml (solver.py:62-65)."""
        spec = PropagationSpec.from_config(self.config, model, npml=self.config.npml)
        check_stability(model, spec)
        return spec

    def components(self, n_components: int = 1) -> tuple[str, ...]:
        if self.config.engine in ("acoustic", "viscoacoustic"):
            return ("p",)
        if int(n_components) >= 4:
            return ("p", "vx", "vz", "sxz")
        return ("vz",)

    def report(self, model: Any) -> dict[str, float]:
        return stability_report(model, self.spec(model))

    def forward(self, model: Any, source: Any, receivers: Any, *, components: tuple[str, ...] | None = None,
                wavelet: np.ndarray | None = None) -> ShotRecord:
        try:
            model.validate()
        except ValueError as exc:
            raise SolverError(f"invalid forward-modelling model: {exc}") from exc
        spec = self.spec(model)
        names = components or self.components()
        record = forward_shot(model, source, receivers, spec, engine=self.config.engine, components=names,
                              q_options=self.q_options())
        record.meta.update({"placeholder": False, "solver": self.name, "engine": self.config.engine,
                            "order": self.config.order, "boundary": self.config.boundary,
                            "npml": self.config.npml, "dt": spec.dt, "nt": spec.nt, "components": list(names)})
        return record

    def wavelet(self, source: Any, model: Any) -> np.ndarray:
        spec = self.spec(model)
        return source_wavelet(source, spec.dt, spec.nt)

    def adjoint(self, record: ShotRecord, model: Any) -> np.ndarray:
        raise SolverError("use RTMImager.migrate for the adjoint (back-propagation and imaging)")


def build_solver(config: SolverConfig, q_config: QConfig | None = None) -> FiniteDifferenceSolver:
    return FiniteDifferenceSolver(config, q_config)
