"""The configuration sections the hot path reads (ertm/config.py:283-436).

Same field names, defaults and validation rules as the reference, so a
reference ``SolverConfig``/``ImagingConfig``/``QConfig`` can be passed
instead of these.
"""

from __future__ import annotations

from dataclasses import dataclass

from .exceptions import ConfigError

_ORDERS = {2, 4, 6, 8}
_BOUNDARIES = {"cpml", "free", "none"}
_DTYPES = {"float32", "float64"}
_ENGINES = {"acoustic", "elastic", "viscoacoustic"}
_MODES = {"pp", "ps", "sp", "ss"}
_CONDITIONS = {"zero_lag", "normalized", "excitation"}
_SEPARATIONS = {"divcurl", "stress"}


@dataclass(frozen=True)
class SolverConfig:
    nt: int = 1200
    dt: float = 5.0e-4
    order: int = 8
    boundary: str = "cpml"
    dtype: str = "float32"
    engine: str = "acoustic"
    npml: int = 20

    def validate(self) -> None:
        if self.nt < 1:
            raise ConfigError("solver.nt must be at least 1")
        if self.dt <= 0:
            raise ConfigError("solver.dt must be positive")
        if self.order not in _ORDERS:
            raise ConfigError(f"solver.order must be one of {sorted(_ORDERS)}")
        if self.boundary not in _BOUNDARIES:
            raise ConfigError(f"solver.boundary must be one of {sorted(_BOUNDARIES)}")
        if self.dtype not in _DTYPES:
            raise ConfigError(f"solver.dtype must be one of {sorted(_DTYPES)}")
        if self.engine not in _ENGINES:
            raise ConfigError(f"solver.engine must be one of {sorted(_ENGINES)}")
        if self.npml < 3:
            raise ConfigError(f"solver.npml must be at least 3, got {self.npml}")


@dataclass(frozen=True)
class ImagingConfig:
    mode: str = "pp"
    condition: str = "normalized"
    separation: str = "divcurl"
    normalize: bool = True
    illumination: bool = True
    receiver_normalization: bool = False
    laplacian: bool = True
    lowpass_fraction: float = 0.85
    checkpoint_mb: float = 256.0
    eps: float = 1.0e-10
    stack_normalize: bool = True
    start_periods: float = 1.5

    def validate(self) -> None:
        if self.mode not in _MODES:
            raise ConfigError(f"imaging.mode must be one of {sorted(_MODES)}")
        if self.condition not in _CONDITIONS:
            raise ConfigError(f"imaging.condition must be one of {sorted(_CONDITIONS)}")
        if self.separation not in _SEPARATIONS:
            raise ConfigError(f"imaging.separation must be one of {sorted(_SEPARATIONS)}")
        if not 0.0 < self.lowpass_fraction <= 1.0:
            raise ConfigError("imaging.lowpass_fraction must lie in (0, 1]")
        if self.checkpoint_mb <= 0:
            raise ConfigError("imaging.checkpoint_mb must be positive")
        if self.eps <= 0:
            raise ConfigError("imaging.eps must be positive")
        if self.start_periods < 0:
            raise ConfigError("imaging.start_periods must not be negative")


@dataclass(frozen=True)
class QConfig:
    enabled: bool = False
    model: str = "filter"
    alpha_c: float = 0.8
    f_ref: float = 30.0
    gain_cap: float = 30.0
    apply_attenuation: bool = False
    attenuation_strength: float = 1.0
    n_mechanisms: int = 3
    band_ratio: float = 1.5
    amplitude_cap: float = 50.0
    lowpass_interval: int = 20
    f_max: float | None = None
    gain_budget_db: float = 40.0
    compare: bool = False

    def validate(self) -> None:
        if not 0.0 <= self.alpha_c <= 1.0:
            raise ConfigError("q.alpha_c must lie in [0, 1]")
        if self.f_ref <= 0:
            raise ConfigError("q.f_ref must be positive")
        if self.gain_cap < 1.0:
            raise ConfigError("q.gain_cap must be at least 1")
        if not 0.0 <= self.attenuation_strength <= 1.0:
            raise ConfigError("q.attenuation_strength must lie in [0, 1]")
        if self.model not in {"filter", "gsls"}:
            raise ConfigError(f"q.model must be filter or gsls, got {self.model!r}")
        if self.n_mechanisms < 1:
            raise ConfigError("q.n_mechanisms must be at least 1")
        if self.band_ratio <= 1.0:
            raise ConfigError("q.band_ratio must exceed 1")
        if self.amplitude_cap < 1.0:
            raise ConfigError("q.amplitude_cap must be at least 1")
        if self.lowpass_interval < 1:
            raise ConfigError("q.lowpass_interval must be at least 1")
        if self.f_max is not None and self.f_max <= 0:
            raise ConfigError("q.f_max must be positive or None")
        if not 0.0 < self.gain_budget_db <= 200.0:
            raise ConfigError("q.gain_budget_db must lie in (0, 200]")
