"""Device propagators with the reference's interface (ertm/propagation.py).

``AcousticPropagator``, ``ViscoacousticPropagator`` and ``ElasticPropagator``
keep the reference's constructor, ``step/sample/inject/image_fields/state/
load_state/state_bytes/reset`` methods and field attributes; the fields,
CPML memories and coefficients live in B200 HBM and every step runs as
sm_100a kernels.  Differences a caller can see:

* field attributes (``prop.p`` …) are read-only host copies, not views;
* wavefields are float32 only (``PropagationSpec.dtype='float64'`` raises
  ``SolverError``) — the FP64 reference is the CPU oracle;
* ``state()`` returns the reference's keys and shapes (ψ expanded to the
  full padded grid), read back from the device.
"""

from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass
from typing import Any

import numpy as np

from . import _lib
from . import numerics as num
from .exceptions import SolverError
from .types import ShotRecord
from .viscoelastic import relaxation_tables


# ---------------------------------------------------------------------------
# spec / stability — propagation.py:44-159
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class PropagationSpec:
    dt: float
    nt: int
    order: int = 8
    npml: int = 20
    dtype: str = "float32"
    boundary: str = "cpml"

    def __post_init__(self) -> None:
        if self.dt <= 0:
            raise ValueError(f"dt must be positive, got {self.dt}")
        if self.nt < 1:
            raise ValueError(f"nt must be at least 1, got {self.nt}")
        if self.order not in num.SUPPORTED_ORDERS:
            raise ValueError(f"order must be one of {num.SUPPORTED_ORDERS}, got {self.order}")
        if self.npml < 1:
            raise ValueError(f"npml must be at least 1, got {self.npml}")
        if self.boundary not in {"cpml", "free", "none"}:
            raise ValueError(f"boundary must be cpml/free/none, got {self.boundary!r}")

    @property
    def numpy_dtype(self) -> np.dtype:
        return np.dtype(self.dtype)

    @property
    def time(self) -> np.ndarray:
        return np.arange(self.nt, dtype=np.float64) * self.dt

    @classmethod
    def from_config(cls, config: Any, model: Any = None, *, npml: int | None = None) -> "PropagationSpec":
        """npml defaults to min(20, max(8, min(nx, nz)//8)) when not passed (propagation.py:84-87)."""
        cells = 20 if model is None else int(min(20, max(8, min(model.grid.nx, model.grid.nz) // 8)))
        return cls(dt=float(config.dt), nt=int(config.nt), order=int(config.order),
                   npml=int(npml if npml is not None else cells), dtype=str(config.dtype),
                   boundary=str(config.boundary))


def stability_report(model: Any, spec: PropagationSpec) -> dict[str, float]:
    vmax = float(np.max(model.vp))
    vmin = float(np.min(model.vp))
    limit = num.cfl_dt(vmax, model.grid.dx, model.grid.dz, spec.order)
    return {"vmax": vmax, "vmin": vmin, "dt": spec.dt, "dt_max": limit,
            "cfl_ratio": float(spec.dt / limit) if limit > 0 else float("inf"),
            "ppw_vmin": num.points_per_wavelength(vmin, 1.0 / (4.0 * spec.dt), model.grid.dx)}


def check_stability(model: Any, spec: PropagationSpec, *, safety: float = 0.55) -> None:
    """Raise SolverError when dt exceeds the CFL limit (propagation.py:113-127)."""
    vmax = float(np.max(model.vp))
    limit = num.cfl_dt(vmax, model.grid.dx, model.grid.dz, spec.order, safety=safety)
    if spec.dt > limit:
        suggested = num.cfl_dt(vmax, model.grid.dx, model.grid.dz, spec.order, safety=0.5)
        raise SolverError(
            f"dt={spec.dt:.3e} s exceeds the CFL limit {limit:.3e} s (vmax={vmax:.0f} m/s, "
            f"dx={model.grid.dx}, dz={model.grid.dz}, order={spec.order}); resample the data to "
            f"dt <= {suggested:.3e} s first.")


@dataclass(frozen=True)
class QOptions:
    enabled: bool = False
    f_ref: float = 30.0
    n_mechanisms: int = 3
    band_ratio: float = 1.5
    compensation: bool = False
    alpha_c: float = 1.0
    amplitude_cap: float = 50.0
    lowpass_interval: int = 20
    f_max: float | None = None
    gain_budget_db: float = 40.0

    def validate(self) -> None:
        if self.f_ref <= 0:
            raise ValueError("q.f_ref must be positive")
        if int(self.n_mechanisms) < 1:
            raise ValueError("q.n_mechanisms must be at least 1")
        if self.band_ratio <= 1.0:
            raise ValueError("q.band_ratio must exceed 1")
        if not 0.0 <= self.alpha_c <= 1.0:
            raise ValueError("q.alpha_c must lie in [0, 1]")
        if self.amplitude_cap < 1.0:
            raise ValueError("q.amplitude_cap must be at least 1")
        if self.f_max is not None and self.f_max <= 0:
            raise ValueError("q.f_max must be positive or None")
        if not 0.0 < self.gain_budget_db <= 200.0:
            raise ValueError("q.gain_budget_db must lie in (0, 200]")


# ---------------------------------------------------------------------------
# propagators
# ---------------------------------------------------------------------------
_OFFSETS = {"vx": (-0.5, 0.0), "vz": (0.0, -0.5), "sxz": (-0.5, -0.5)}


class _PMLView:
    """What the reference exposes as ``prop.pml`` (lazy ψ bookkeeping only)."""

    def __init__(self, prop: "Propagator2D") -> None:
        self._prop = weakref.ref(prop)

    @property
    def _memory(self) -> dict[str, None]:
        p = self._prop()
        return {k: None for k in p._psi_terms} if p is not None and p._psi_allocated else {}

    def memory_bytes(self) -> int:
        p = self._prop()
        if p is None or not p._psi_allocated:
            return 0
        return len(p._psi_terms) * p.shape[0] * p.shape[1] * 4


class Propagator2D:
    """Common part: geometry, CPML strips, device handle, state I/O."""

    name = "propagator-2d"
    components: tuple[str, ...] = ()
    _field_slots: dict[str, int] = {}
    _psi_terms: dict[str, tuple[int, int]] = {}   # name → (axis, term)
    _engine = "acoustic"

    def __init__(self, model: Any, spec: PropagationSpec, *, q_options: QOptions | None = None,
                 stream: int | None = None) -> None:
        if hasattr(model, "validate"):
            model.validate()
        if np.dtype(spec.dtype) != np.float32:
            raise SolverError("the B200 path propagates float32 wavefields only (dtype='float32')")
        self.model = model
        self.spec = spec
        self.grid = model.grid
        self.dt = float(spec.dt)
        self.nt = int(spec.nt)
        self.order = int(spec.order)
        self.coeffs = num.staggered_coefficients(self.order)
        self.pad = num.ghost_width(self.order)
        self.dtype = np.dtype(np.float32)
        self.shape = (self.grid.nz + 2 * self.pad, self.grid.nx + 2 * self.pad)
        self.dx, self.dz = float(self.grid.dx), float(self.grid.dz)
        self.x0, self.z0 = float(getattr(self.grid, "x0", 0.0)), float(getattr(self.grid, "z0", 0.0))
        self._source_index: tuple[int, int] | None = None
        self._source = None
        self._mechanism = "explosive"
        self._receivers = None
        self._psi_allocated = False
        self.pml = _PMLView(self)
        self._handle = None
        self._stream = stream
        self._create(model, q_options)

    # ---------------------------------------------------------------- set-up
    def _strips(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray, tuple[int, int, int, int]]:
        """CPML profiles of the padded axes (propagation.py:221-235)."""
        nzp, nxp = self.shape
        vmax = float(np.max(self.model.vp))
        enabled = self.spec.boundary != "none"
        top = self.spec.boundary != "free"
        amax = 2.0 * np.pi * float(max(25.0, 1.0))
        bx, ax, nx_ = num.cpml_profile(nxp, self.dx, self.spec.npml, self.dt, vmax, alpha_max=amax,
                                       enabled=enabled)
        bz, az, nz_ = num.cpml_profile(nzp, self.dz, self.spec.npml, self.dt, vmax, alpha_max=amax,
                                       sides=(top, True), enabled=enabled)
        widths = (nx_, nx_, nz_ if top else 0, nz_) if enabled else (0, 0, 0, 0)
        return ax, bx, az, bz, widths

    def _create(self, model: Any, q: QOptions | None) -> None:
        L = _lib.lib()
        ax, bx, az, bz, (xl, xr, zt, zb) = self._strips()
        cfg = _lib.PropConfig()
        cfg.engine = _lib.ENGINE[self._engine]
        cfg.order = self.order
        cfg.nx, cfg.nz = self.grid.nx, self.grid.nz
        cfg.dx, cfg.dz, cfg.x0, cfg.z0, cfg.dt = self.dx, self.dz, self.x0, self.z0, self.dt
        cfg.free_surface = 1 if self.spec.boundary == "free" else 0
        cfg.npml_x_left, cfg.npml_x_right, cfg.npml_z_top, cfg.npml_z_bottom = xl, xr, zt, zb
        vp = np.ascontiguousarray(model.vp, dtype=np.float32)
        rho = np.ascontiguousarray(model.rho, dtype=np.float32)
        vs = np.ascontiguousarray(model.vs, dtype=np.float32)
        tables = self._tables(cfg)
        keep = [vp, rho, vs, ax, bx, az, bz]
        args = [None] * 5
        if tables is not None:
            args = [tables.qidx, tables.tau, tables.delta, tables.modulus_ref, tables.relax_a]
            keep += args
        h = L.ertm_prop_create(cfg, _lib.ptr(vp), _lib.ptr(vs), _lib.ptr(rho), _lib.ptr(ax), _lib.ptr(bx),
                               _lib.ptr(az), _lib.ptr(bz), *[_lib.ptr(a) for a in args], self._stream)
        if not h:
            raise SolverError(f"device propagator creation failed: {_lib.last_error()}")
        self._handle = h
        self._finalizer = weakref.finalize(self, L.ertm_prop_destroy, h)
        self._info_cache = self.info()

    def _tables(self, cfg: _lib.PropConfig):
        return None

    @property
    def handle(self) -> int:
        return self._handle

    def info(self) -> _lib.PropInfo:
        info = _lib.PropInfo()
        _lib.check(_lib.lib().ertm_prop_info_get(self._handle, info), "info")
        return info

    @property
    def step_index(self) -> int:
        return int(self.info().step_index)

    @step_index.setter
    def step_index(self, value: int) -> None:
        _lib.check(_lib.lib().ertm_prop_set_step_index(self._handle, int(value)), "set_step_index")

    # --------------------------------------------------------------- geometry
    def node_index(self, x: float, z: float) -> tuple[int, int]:
        """propagation.py:246-249 (round half to even, clipped to the grid)."""
        ix = min(max(int(round((float(x) - self.x0) / self.dx)), 0), self.grid.nx - 1)
        iz = min(max(int(round((float(z) - self.z0) / self.dz)), 0), self.grid.nz - 1)
        return iz + self.pad, ix + self.pad

    def fractional_index(self, x, z, *, x_offset: float = 0.0, z_offset: float = 0.0):
        xf = (np.asarray(x, dtype=np.float64) - self.x0) / self.dx + self.pad + x_offset
        zf = (np.asarray(z, dtype=np.float64) - self.z0) / self.dz + self.pad + z_offset
        return zf, xf

    def set_source(self, source: Any) -> None:
        self._source_index = self.node_index(source.x, source.z)
        self._source = source
        self._mechanism = str(getattr(source, "mechanism", "explosive"))
        iz, ix = self._source_index
        _lib.check(_lib.lib().ertm_prop_set_source(self._handle, iz, ix, _lib.MECH[self._mechanism]),
                   "set_source")

    def set_receivers(self, receivers: Any) -> None:
        self._receivers = receivers
        x = np.ascontiguousarray(np.asarray(receivers.x, dtype=np.float64).reshape(-1))
        z = np.ascontiguousarray(np.asarray(receivers.z, dtype=np.float64).reshape(-1))
        _lib.check(_lib.lib().ertm_prop_set_receivers(self._handle, x.size, _lib.ptr(x), _lib.ptr(z)),
                   "set_receivers")

    # ------------------------------------------------------------- state I/O
    def _field_names(self) -> tuple[str, ...]:
        return tuple(self._field_slots)

    def _read(self, slot: int) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float32)
        _lib.check(_lib.lib().ertm_prop_read_field(self._handle, slot, _lib.ptr(out)), "read_field")
        return out

    def _write(self, slot: int, value: np.ndarray) -> None:
        arr = np.ascontiguousarray(np.broadcast_to(np.asarray(value, dtype=np.float32), self.shape))
        _lib.check(_lib.lib().ertm_prop_write_field(self._handle, slot, _lib.ptr(arr)), "write_field")

    def _get(self, name: str) -> np.ndarray:
        return self._read(self._field_slots[name])

    def __getattr__(self, name: str):
        slots = type(self)._field_slots
        if name in slots and "_handle" in self.__dict__:
            return self._get(name)
        raise AttributeError(name)

    def _crop(self, field: np.ndarray) -> np.ndarray:
        lo = self.pad
        return field[lo: lo + self.grid.nz, lo: lo + self.grid.nx]

    def state(self) -> dict[str, np.ndarray]:
        """Fields, CPML memories (after the first step) and the step counter (propagation.py:283-289)."""
        s = {n: self._get(n) for n in self._field_names()}
        if self._psi_allocated:
            for key, (axis, term) in self._psi_terms.items():
                out = np.empty(self.shape, dtype=np.float32)
                _lib.check(_lib.lib().ertm_prop_read_psi(self._handle, axis, term, _lib.ptr(out)), "read_psi")
                s[f"pml:{key}"] = out
        s["_step"] = np.array(self.step_index, dtype=np.int64)
        return s

    def load_state(self, state: dict[str, np.ndarray]) -> None:
        """propagation.py:291-299: CPML memories are restored only once they exist."""
        for name in self._field_names():
            self._set_field(name, state[name])
        if self._psi_allocated:
            for key, (axis, term) in self._psi_terms.items():
                cached = state.get(f"pml:{key}")
                if cached is not None:
                    arr = np.ascontiguousarray(cached, dtype=np.float32)
                    _lib.check(_lib.lib().ertm_prop_write_psi(self._handle, axis, term, _lib.ptr(arr)),
                               "write_psi")
        self.step_index = int(np.asarray(state["_step"]).item())

    def _set_field(self, name: str, value: np.ndarray) -> None:
        self._write(self._field_slots[name], value)

    def state_bytes(self) -> int:
        """Reference accounting: padded fields + CPML memories once allocated (propagation.py:301-306)."""
        return int(self._info_cache.field_bytes + self.pml.memory_bytes())

    def device_state_bytes(self) -> int:
        """Bytes one device checkpoint actually takes (fields + CPML strips only)."""
        return int(self._info_cache.state_bytes)

    def reset(self) -> None:
        _lib.check(_lib.lib().ertm_prop_reset(self._handle), "reset")
        self._psi_allocated = False

    # ------------------------------------------------------------- interface
    def step(self, source_amplitude: float = 0.0) -> None:
        amp = np.array([float(source_amplitude)], dtype=np.float64)
        _lib.check(_lib.lib().ertm_prop_step(self._handle, 1, _lib.ptr(amp)), "step")
        self._psi_allocated = True

    @property
    def status(self) -> int:
        """Device status bits after the queued steps (no reference counterpart):
        bit 0 set once a step wrote NaN or infinity into a wavefield."""
        out = C.c_uint32()
        _lib.check(_lib.lib().ertm_prop_status(self._handle, C.byref(out)), "status")
        return int(out.value)

    @property
    def finite(self) -> bool:
        return not (self.status & _lib.STATUS_NONFINITE)

    def run(self, amplitudes: np.ndarray) -> None:
        """Advance len(amplitudes) steps in one call (no reference counterpart)."""
        amps = np.ascontiguousarray(amplitudes, dtype=np.float64)
        _lib.check(_lib.lib().ertm_prop_step(self._handle, amps.size, _lib.ptr(amps)), "step")
        if amps.size:
            self._psi_allocated = True

    def _check_component(self, name: str, action: str) -> int:
        raise NotImplementedError

    def sample(self, components: tuple[str, ...] | None = None) -> dict[str, np.ndarray]:
        if self._receivers is None:
            return {}
        names = tuple(components or self._default_sample)
        codes = np.array([self._check_component(n, "sample") for n in names], dtype=np.int32)
        out = np.empty((len(names), int(np.asarray(self._receivers.x).size)), dtype=np.float32)
        _lib.check(_lib.lib().ertm_prop_sample(self._handle, len(names), _lib.ptr(codes), _lib.ptr(out)),
                   "sample")
        return {n: out[i] for i, n in enumerate(names)}

    def inject(self, component: str, values: np.ndarray) -> None:
        if self._receivers is None:
            raise SolverError("receivers must be set before injecting data")
        code = self._check_component(component, "inject")
        v = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
        _lib.check(_lib.lib().ertm_prop_inject(self._handle, code, _lib.ptr(v)), "inject")

    def _image(self, wave: str, separation: str) -> np.ndarray:
        out = np.empty(self.grid.shape, dtype=np.float32)
        _lib.check(_lib.lib().ertm_prop_image_field(self._handle, _lib.WAVE[wave], _lib.SEP.get(separation, 0),
                                                   _lib.ptr(out)), "image_field")
        return out

    def image_fields(self, separation: str = "stress") -> dict[str, np.ndarray]:
        return {"P": self._image("P", "stress")}


class AcousticPropagator(Propagator2D):
    """Velocity–pressure engine (propagation.py:397-504)."""

    name = "acoustic-velocity-pressure"
    components = ("p", "vx", "vz")
    _engine = "acoustic"
    _field_slots = {"p": 0, "vx": 1, "vz": 2}
    _psi_terms = {"vx_dp_dx": (1, 0), "vz_dp_dz": (0, 0), "p_dvx_dx": (1, 1), "p_dvz_dz": (0, 1)}
    _default_sample = ("p",)

    def _check_component(self, name: str, action: str) -> int:
        if action == "sample" and name == "sxz":
            return _lib.COMP["sxz"]   # sampled as zeros (propagation.py:464-466)
        if name not in self.components:
            verb = "sample" if action == "sample" else "inject"
            raise SolverError(f"acoustic propagator cannot {verb} component {name!r}; options {self.components}")
        return _lib.COMP[name]

    @property
    def max_amplitude(self) -> float:
        return float(np.max(np.abs(self.p)))


class ViscoacousticPropagator(Propagator2D):
    """GSLS viscoacoustic engine (propagation.py:510-797)."""

    name = "viscoacoustic-gsls"
    components = ("p", "vx", "vz")
    _engine = "viscoacoustic"
    _psi_terms = {"vx_dp_dx": (1, 0), "vz_dp_dz": (0, 0), "p_dvx_dx": (1, 1), "p_dvz_dz": (0, 1)}
    _default_sample = ("p",)

    def __init__(self, model: Any, spec: PropagationSpec, *, q_options: QOptions | None = None,
                 stream: int | None = None) -> None:
        self.q_options = q_options or QOptions(enabled=True)
        self.q_options.validate()
        super().__init__(model, spec, q_options=self.q_options, stream=stream)

    @property
    def _field_slots(self) -> dict[str, int]:  # type: ignore[override]
        return {"p": 0, "vx": 1, "vz": 2, "eps": 3}

    def _field_names(self) -> tuple[str, ...]:
        return ("p", "vx", "vz", "eps", "r")

    def _get(self, name: str) -> np.ndarray:
        if name == "r":
            return np.stack([self._read(4 + l) for l in range(self.n_mechanisms)])
        return self._read({"p": 0, "vx": 1, "vz": 2, "eps": 3}[name])

    def _set_field(self, name: str, value: np.ndarray) -> None:
        if name == "r":
            arr = np.asarray(value, dtype=np.float32)
            for l in range(self.n_mechanisms):
                self._write(4 + l, arr[l])
        else:
            self._write({"p": 0, "vx": 1, "vz": 2, "eps": 3}[name], value)

    def __getattr__(self, name: str):
        if name in ("p", "vx", "vz", "eps", "r") and "_handle" in self.__dict__:
            return self._get(name)
        raise AttributeError(name)

    def _tables(self, cfg: _lib.PropConfig):
        q = self.q_options
        qp = np.pad(np.asarray(self.model.qp).astype(np.float32, copy=False), self.pad, mode="edge")
        t = relaxation_tables(qp, self.dt, self.nt, f_ref=q.f_ref, n_mechanisms=int(q.n_mechanisms),
                              band_ratio=q.band_ratio, compensation=bool(q.compensation), alpha_c=q.alpha_c,
                              f_max=q.f_max, gain_budget_db=q.gain_budget_db)
        self.n_mechanisms = int(q.n_mechanisms)
        self.q_fit_error = float(t.fit_error)
        self.alpha_mechanisms = t.alpha_mechanisms
        self.f_peak_mechanisms = t.f_peak_mechanisms
        self.relaxation = t
        cfg.n_mech = self.n_mechanisms
        cfg.n_q = int(t.q_values.size)
        cfg.compensation = 1 if q.compensation else 0
        cfg.amplitude_cap = float(q.amplitude_cap)
        cfg.lowpass_interval = int(q.lowpass_interval)
        t.qidx = np.ascontiguousarray(t.qidx)
        t.tau = np.ascontiguousarray(t.tau)
        t.delta = np.ascontiguousarray(t.delta)
        t.modulus_ref = np.ascontiguousarray(t.modulus_ref)
        t.relax_a = np.ascontiguousarray(t.relax_a)
        return t

    def state_bytes(self) -> int:
        info = self._info_cache
        return int(info.field_bytes + self.pml.memory_bytes())

    def inject(self, component: str, values: np.ndarray) -> None:
        if self._receivers is None:
            raise SolverError("receivers must be set before injecting data")
        super().inject(component, values)

    def _check_component(self, name: str, action: str) -> int:
        if name not in self.components:
            verb = "sample" if action == "sample" else "inject"
            raise SolverError(f"viscoacoustic propagator cannot {verb} component {name!r}")
        return _lib.COMP[name]

    @property
    def quality_summary(self) -> dict[str, Any]:
        info = self.info()
        return {
            "mechanisms": int(self.n_mechanisms),
            "q_fit_error": float(self.q_fit_error),
            "compensation": bool(self.q_options.compensation),
            "alpha_c": float(self.q_options.alpha_c),
            "alpha_mechanisms": list(self.alpha_mechanisms),
            "f_peak_mechanisms_hz": [round(v, 1) for v in self.f_peak_mechanisms],
            "f_max": None if self.q_options.f_max is None else float(self.q_options.f_max),
            "gain_budget_db": float(self.q_options.gain_budget_db),
            "clipped": int(info.clipped),
            "lowpass_steps": int(info.lowpass_steps),
        }


class ElasticPropagator(Propagator2D):
    """P-SV velocity–stress engine (propagation.py:803-980)."""

    name = "elastic-velocity-stress"
    components = ("vx", "vz", "sxx", "szz", "sxz", "p")
    _engine = "elastic"
    _field_slots = {"vx": 0, "vz": 1, "sxx": 2, "szz": 3, "sxz": 4}
    _psi_terms = {"vx_dsxx": (1, 0), "vx_dsxz": (0, 0), "vz_dsxz": (1, 1), "vz_dszz": (0, 1),
                  "sxx_dvx": (1, 2), "szz_dvz": (0, 2), "sxz_dvx": (0, 3), "sxz_dvz": (1, 3)}
    _default_sample = ("vx", "vz")

    def _check_component(self, name: str, action: str) -> int:
        if name not in _lib.COMP:
            verb = "sample" if action == "sample" else "inject"
            raise SolverError(f"elastic propagator cannot {verb} component {name!r}; options {self.components}")
        return _lib.COMP[name]

    def pressure_field(self) -> np.ndarray:
        return 0.5 * (self.sxx + self.szz)

    def shear_field(self) -> np.ndarray:
        return self.sxz

    def image_fields(self, separation: str = "stress") -> dict[str, np.ndarray]:
        mode = str(separation).lower()
        if mode not in ("stress", "divcurl"):
            raise SolverError(f"unknown P/S separation {separation!r}; choose stress/divcurl")
        return {"P": self._image("P", mode), "S": self._image("S", mode)}


def build_propagator(model: Any, spec: PropagationSpec, *, engine: str = "acoustic",
                     q_options: QOptions | None = None, stream: int | None = None) -> Propagator2D:
    """propagation.py:986-1001."""
    engine = str(engine).lower()
    if engine == "acoustic":
        return AcousticPropagator(model, spec, stream=stream)
    if engine == "viscoacoustic":
        return ViscoacousticPropagator(model, spec, q_options=q_options, stream=stream)
    if engine == "elastic":
        return ElasticPropagator(model, spec, stream=stream)
    raise SolverError(f"unknown engine {engine!r}; choose acoustic/viscoacoustic/elastic")


def source_wavelet(source: Any, dt: float, nt: int) -> np.ndarray:
    """propagation.py:1004-1015."""
    t = np.arange(nt, dtype=np.float64) * dt
    kind = getattr(source, "kind", "ricker")
    if kind == "ricker":
        wave = num.ricker(t, source.f0, source.delay)
    elif kind == "gaussian":
        wave = num.gaussian_pulse(t, source.f0, source.delay)
    elif kind == "custom":
        raise SolverError("a custom source needs an explicit time series")
    else:
        raise SolverError(f"unsupported source kind: {kind}")
    return (float(getattr(source, "amplitude", 1.0)) * wave).astype(np.float32)


def run_forward(model: Any, source: Any, receivers: Any, spec: PropagationSpec, *, engine: str = "acoustic",
                components: tuple[str, ...] | None = None, wavelet: np.ndarray | None = None,
                propagator: Propagator2D | None = None, record_every: int = 1,
                q_options: QOptions | None = None) -> dict[str, np.ndarray]:
    """Forward modelling in one device call (propagation.py:1018-1052)."""
    prop = propagator or build_propagator(model, spec, engine=engine, q_options=q_options)
    prop.set_source(source)
    prop.set_receivers(receivers)
    if wavelet is None:
        wavelet = source_wavelet(source, spec.dt, spec.nt)
    w = np.ascontiguousarray(wavelet, dtype=np.float32)
    nt = int(w.size)
    names = tuple(components or prop.components[:1])
    codes = np.array([prop._check_component(n, "sample") for n in names], dtype=np.int32)
    nrec = int(np.asarray(receivers.x).size)
    out = np.zeros((len(names), nt, nrec), dtype=np.float32)
    _lib.check(_lib.lib().ertm_forward(prop.handle, nt, _lib.ptr(w), len(names), _lib.ptr(codes), _lib.ptr(out)),
               "forward")
    if nt:
        prop._psi_allocated = True
    if record_every > 1:
        out[:, np.arange(nt) % record_every != 0, :] = 0.0
    return {n: out[i] for i, n in enumerate(names)}


def forward_shot(model: Any, source: Any, receivers: Any, spec: PropagationSpec, *, engine: str = "acoustic",
                 components: tuple[str, ...] | None = None, q_options: QOptions | None = None) -> ShotRecord:
    """propagation.py:1055-1093."""
    names = components or (("p",) if engine in ("acoustic", "viscoacoustic") else ("vx", "vz", "sxz"))
    data = run_forward(model, source, receivers, spec, engine=engine, components=names, q_options=q_options)
    primary = names[0]
    t = np.arange(data[primary].shape[0], dtype=np.float64) * spec.dt
    meta = {"engine": engine, "solver": f"{engine}-velocity-stress", "dt": spec.dt, "nt": int(t.size),
            "order": spec.order, "npml": spec.npml, "components": list(names), "placeholder": False,
            "method": "finite-difference two-way wave equation", "device": "B200 (sm_100a)"}
    shot = ShotRecord(data=data[primary].astype(np.float32), dt=float(spec.dt), t=t, receivers=receivers,
                      source=source, meta=meta, components={n: data[n].astype(np.float32) for n in names})
    shot.validate()
    return shot
