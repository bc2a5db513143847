"""Data contracts with the reference's field names (ertm/types.py:20-265).

The GPU path accepts these or the reference's own objects (duck typing on
the attribute names); arrays are ``(nz, nx)`` C-order, time series
``(nt, nrec)``.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np


@dataclass(frozen=True)
class GridSpec:
    nx: int
    nz: int
    dx: float
    dz: float
    x0: float = 0.0
    z0: float = 0.0

    def __post_init__(self) -> None:
        if self.nx < 2 or self.nz < 2:
            raise ValueError(f"grid needs at least 2x2 cells, got {self.nx}x{self.nz}")
        if self.dx <= 0 or self.dz <= 0:
            raise ValueError(f"grid spacing must be positive, got dx={self.dx}, dz={self.dz}")

    @property
    def shape(self) -> tuple[int, int]:
        return (self.nz, self.nx)

    @property
    def size(self) -> int:
        return self.nx * self.nz

    @property
    def x_min(self) -> float:
        return float(self.x0)

    @property
    def x_max(self) -> float:
        return float(self.x0 + (self.nx - 1) * self.dx)

    @property
    def z_min(self) -> float:
        return float(self.z0)

    @property
    def z_max(self) -> float:
        return float(self.z0 + (self.nz - 1) * self.dz)

    def x_at(self, ix: int) -> float:
        return float(self.x0 + ix * self.dx)

    def z_at(self, iz: int) -> float:
        return float(self.z0 + iz * self.dz)

    def index_of(self, x: float, z: float, *, clip: bool = True) -> tuple[int, int]:
        """Nearest node ``(ix, iz)``; Python's round (half to even) as in types.py:73-82."""
        ix = int(round((float(x) - self.x0) / self.dx))
        iz = int(round((float(z) - self.z0) / self.dz))
        if clip:
            return min(max(ix, 0), self.nx - 1), min(max(iz, 0), self.nz - 1)
        if not (0 <= ix < self.nx and 0 <= iz < self.nz):
            raise ValueError(f"point ({x}, {z}) lies outside the grid")
        return ix, iz


@dataclass
class ElasticModel:
    grid: GridSpec
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    qp: np.ndarray
    qs: np.ndarray
    name: str = "model"
    meta: dict[str, Any] = field(default_factory=dict)

    @property
    def shape(self) -> tuple[int, int]:
        return self.grid.shape

    def validate(self) -> "ElasticModel":
        """Shapes, finiteness, positivity and vs < vp (types.py:106-122)."""
        for key in ("vp", "vs", "rho", "qp", "qs"):
            value = getattr(self, key)
            if not isinstance(value, np.ndarray):
                raise ValueError(f"model field {key} must be a numpy array")
            if value.shape != self.shape:
                raise ValueError(f"model field {key} has shape {value.shape}, grid is {self.shape}")
            if not np.all(np.isfinite(value)):
                raise ValueError(f"model field {key} contains NaN/Inf")
            if np.any(value <= 0):
                raise ValueError(f"model field {key} must be positive")
        if np.any(self.vs >= self.vp):
            raise ValueError("model must satisfy vs < vp")
        return self


@dataclass(frozen=True)
class SourceSpec:
    x: float
    z: float
    f0: float = 20.0
    kind: str = "ricker"
    amplitude: float = 1.0
    delay: float = 0.0
    mechanism: str = "explosive"

    def __post_init__(self) -> None:
        if self.mechanism not in {"explosive", "shear", "force_z"}:
            raise ValueError(f"source.mechanism must be explosive/shear/force_z, got {self.mechanism!r}")


@dataclass(frozen=True)
class ReceiverSpec:
    x: np.ndarray
    z: np.ndarray
    component: str = "vz"

    def __post_init__(self) -> None:
        x = np.asarray(self.x, dtype=float).reshape(-1)
        z = np.asarray(self.z, dtype=float).reshape(-1)
        if x.size == 0 or z.size == 0:
            raise ValueError("receivers must not be empty")
        if x.size != z.size:
            raise ValueError(f"receiver x/z counts differ: {x.size} vs {z.size}")
        object.__setattr__(self, "x", x)
        object.__setattr__(self, "z", z)

    @property
    def nrec(self) -> int:
        return int(self.x.size)


@dataclass
class ShotRecord:
    data: np.ndarray
    dt: float
    t: np.ndarray
    receivers: ReceiverSpec
    source: SourceSpec
    meta: dict[str, Any] = field(default_factory=dict)
    components: dict[str, np.ndarray] = field(default_factory=dict)

    def validate(self) -> "ShotRecord":
        """types.py:202-224."""
        data = np.asarray(self.data)
        if data.ndim != 2:
            raise ValueError(f"shot record must be 2-D (nt, nrec), got {data.shape}")
        if data.shape[0] != np.asarray(self.t).size:
            raise ValueError("record time axis and t differ in length")
        if data.shape[1] != self.receivers.nrec:
            raise ValueError("record traces and receivers differ in count")
        if self.dt <= 0:
            raise ValueError("dt must be positive")
        if not np.all(np.isfinite(data)):
            raise ValueError("shot record contains NaN/Inf")
        for name, arr in self.components.items():
            comp = np.asarray(arr)
            if comp.shape != data.shape:
                raise ValueError(f"component {name!r} has shape {comp.shape}, primary is {data.shape}")
            if not np.all(np.isfinite(comp)):
                raise ValueError(f"component {name!r} contains NaN/Inf")
        return self

    def component(self, name: str) -> np.ndarray:
        if name in self.components:
            return self.components[name]
        if name == "primary":
            return self.data
        raise KeyError(f"no component {name!r}; available: {sorted(self.components) or ['primary']}")

    @property
    def component_names(self) -> tuple[str, ...]:
        return tuple(self.components) or ("primary",)


@dataclass
class ImageResult:
    image: np.ndarray
    grid: GridSpec
    mode: str = "pp"
    meta: dict[str, Any] = field(default_factory=dict)

    def validate(self) -> "ImageResult":
        image = np.asarray(self.image)
        if image.shape != self.grid.shape:
            raise ValueError(f"image shape {image.shape} differs from grid {self.grid.shape}")
        if not np.all(np.isfinite(image)):
            raise ValueError("image contains NaN/Inf")
        return self
