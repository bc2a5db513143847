"""Reverse-time migration with the reference's interface (ertm/imaging.py).

``RTMImager.migrate`` keeps the reference signature and result; the
checkpointed forward pass, the block replay, the time-reversed record
injection, the backward pass and the imaging condition run in one call of
the CUDA driver (``ertm_migrate``) with every wavefield, checkpoint and
accumulator in HBM.  Normalisation, Laplacian, wavenumber low-pass and the
PML mask run on the device as well (``ertm_postprocess``).
"""

from __future__ import annotations

import threading
import weakref
from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np

from . import _lib
from . import numerics as num
from .config import ImagingConfig, QConfig, SolverConfig
from .exceptions import ImagingError, SolverError
from .propagation import (PropagationSpec, Propagator2D, QOptions, build_propagator, check_stability,
                          source_wavelet)
from .types import ImageResult

#: imaging mode → (source wave, receiver wave) (imaging.py:47-52)
WAVE_MODES: dict[str, tuple[str, str]] = {"pp": ("P", "P"), "ps": ("P", "S"), "sp": ("S", "P"), "ss": ("S", "S")}
_ACOUSTIC_MODES = {"pp"}


def zero_lag_condition(source_wavefield: np.ndarray, receiver_wavefield: np.ndarray) -> np.ndarray:
    """Integrand W_s·W_r of the zero-lag cross-correlation (imaging.py:61-66)."""
    return np.asarray(source_wavefield) * np.asarray(receiver_wavefield)


def normalized_terms(source_wavefield, receiver_wavefield):
    """(W_s·W_r, W_s², W_r²) (imaging.py:69-79)."""
    s, r = np.asarray(source_wavefield), np.asarray(receiver_wavefield)
    return s * r, s * s, r * r


def excitation_terms(source_amplitude, receiver_wavefield):
    """A_s·W_r at the excitation time (imaging.py:82-87)."""
    return np.asarray(source_amplitude) * np.asarray(receiver_wavefield)


@dataclass
class CheckpointStore:
    """Checkpoint bookkeeping (imaging.py:93-110).

    ``states`` holds ``(step, state)`` pairs when filled through the granular
    ``record_source_wavefield``; the device driver keeps its checkpoints in
    HBM and only reports interval and count here.
    """

    states: list = field(default_factory=list)
    interval: int = 1
    bytes_per_state: int = 0
    n_states: int | None = None

    @property
    def memory_mb(self) -> float:
        count = len(self.states) if self.n_states is None else self.n_states
        return count * self.bytes_per_state / (1024.0**2)

    def summary(self) -> dict[str, Any]:
        count = len(self.states) if self.n_states is None else self.n_states
        return {"interval": int(self.interval), "n_states": int(count), "memory_mb": round(self.memory_mb, 3)}


def checkpoint_interval(nt: int, bytes_per_state: int, budget_mb: float) -> int:
    """imaging.py:121-124 — states that fit the budget, then the step between them."""
    per = max(int(bytes_per_state), 1)
    budget = max(float(budget_mb), 1.0) * 1024.0**2
    n_states = max(1, int(budget // per))
    return max(1, int(np.ceil(nt / n_states)))


def record_source_wavefield(prop: Propagator2D, wavelet: np.ndarray, *, budget_mb: float) -> CheckpointStore:
    """Granular form of the checkpointed forward pass (imaging.py:113-137)."""
    nt = int(len(wavelet))
    per = max(int(prop.state_bytes()), 1)
    store = CheckpointStore(interval=checkpoint_interval(nt, per, budget_mb), bytes_per_state=per)
    for step in range(nt):
        prop.step(float(wavelet[step]))
        if step % store.interval == 0:
            store.states.append((step, prop.state()))
    return store


def replay_block(prop: Propagator2D, wavelet: np.ndarray, store: CheckpointStore, block_index: int,
                 separation: str) -> list[dict[str, np.ndarray]]:
    """Granular block replay (imaging.py:140-162): restore, re-run, copy image fields."""
    start, state = store.states[block_index]
    prop.load_state(state)
    end = store.states[block_index + 1][0] if block_index + 1 < len(store.states) else len(wavelet)
    out = []
    for step in range(start, end):
        prop.step(float(wavelet[step]))
        out.append({k: np.array(v, copy=True) for k, v in prop.image_fields(separation).items()})
    return out


def _target_component(name: str, engine: str) -> str:
    """imaging.py:437-444."""
    if name in ("primary", "p") and engine == "acoustic":
        return "p"
    if name == "primary":
        return "vz"
    return name


def postprocess_image(num: np.ndarray, illum: np.ndarray | None, rillum: np.ndarray | None, *, dx: float,
                      dz: float, by_illum: bool, by_rillum: bool, eps: float, laplacian: bool,
                      lowpass_fraction: float, npml: int, boundary: str) -> np.ndarray:
    """Normalisation + Laplacian + low-pass + PML mask on the device (imaging.py:326-333, 476-502)."""
    nz, nx = num.shape
    out = np.empty((nz, nx), dtype=np.float32)
    n64 = np.ascontiguousarray(num, dtype=np.float64)
    i64 = None if illum is None else np.ascontiguousarray(illum, dtype=np.float64)
    r64 = None if rillum is None else np.ascontiguousarray(rillum, dtype=np.float64)
    _lib.check(_lib.lib().ertm_postprocess(nz, nx, float(dx), float(dz), _lib.ptr(n64), _lib.ptr(i64),
                                          _lib.ptr(r64), int(by_illum), int(by_rillum), float(eps),
                                          int(bool(laplacian)), float(lowpass_fraction), int(npml),
                                          int(boundary == "cpml"), _lib.ptr(out), None), "postprocess")
    return out


class RTMImager:
    """Single-shot reverse-time migration (imaging.py:168-563)."""

    name = "rtm-imager"

    def __init__(self, imaging_config: ImagingConfig, solver_config: SolverConfig | None = None,
                 q_config: QConfig | None = None, *, accumulation: str = "fp64") -> None:
        self.config = imaging_config
        self.config.validate()
        self.solver_config = solver_config or SolverConfig()
        self.solver_config.validate()
        self.q_config = q_config or QConfig()
        self.q_config.validate()
        if accumulation not in _lib.ACCUM:
            raise ImagingError(f"accumulation must be one of {sorted(_lib.ACCUM)}")
        self.accumulation = accumulation
        self._validate_engine_mode()
        self._pool = MigratorPool(self)
        self._pool_lock = threading.Lock()

    def q_options(self, *, compensation: bool = False) -> QOptions | None:
        """imaging.py:187-202."""
        if self.solver_config.engine != "viscoacoustic":
            return None
        q = self.q_config
        return QOptions(enabled=True, f_ref=float(q.f_ref), n_mechanisms=int(q.n_mechanisms),
                        band_ratio=float(q.band_ratio), compensation=bool(compensation and q.enabled),
                        alpha_c=float(q.alpha_c), amplitude_cap=float(q.amplitude_cap),
                        lowpass_interval=int(q.lowpass_interval),
                        f_max=None if q.f_max is None else float(q.f_max), gain_budget_db=float(q.gain_budget_db))

    # ------------------------------------------------------------- public API
    def migrate(self, shot: Any, model: Any, *, wavelet: np.ndarray | None = None,
                preprocess: Callable[[np.ndarray, float], np.ndarray] | None = None,
                modes: tuple[str, ...] | None = None) -> ImageResult:
        """Migrate one shot.  ``modes`` (extension) images several wave modes
        from one forward/replay/backward pass; the result then carries the
        extra images in ``meta['images']``."""
        results = self.migrate_modes(shot, model, wavelet=wavelet, preprocess=preprocess,
                                     modes=modes or (self.config.mode,))
        first = results[0]
        if len(results) > 1:
            first.meta["images"] = {r.mode: r.image for r in results}
        return first

    def migrate_modes(self, shot: Any, model: Any, *, wavelet: np.ndarray | None = None,
                      preprocess: Callable | None = None, modes: tuple[str, ...] = ("pp",)) -> list[ImageResult]:
        try:
            shot.validate()
            model.validate()
        except ValueError as exc:
            raise ImagingError(f"invalid imaging input: {exc}") from exc
        # the last model's propagator pair is kept for the next call; a call
        # made while another thread migrates with this imager builds its own
        if not self._pool_lock.acquire(blocking=False):
            return ShotMigrator(self, model).migrate(shot, wavelet=wavelet, preprocess=preprocess, modes=modes)
        try:
            self._pool.begin([model])
            mig = self._pool.take(model, {})
            return mig.migrate(shot, wavelet=wavelet, preprocess=preprocess, modes=modes)
        finally:
            self._pool_lock.release()

    def release(self) -> None:
        """Free the propagator pair kept from the last call."""
        with self._pool_lock:
            self._pool.clear()

    def image_condition(self, source_wavefield: np.ndarray, receiver_wavefield: np.ndarray) -> np.ndarray:
        s, r = np.asarray(source_wavefield), np.asarray(receiver_wavefield)
        if s.shape != r.shape:
            raise ImagingError(f"imaging-condition inputs differ in shape: {s.shape} vs {r.shape}")
        return zero_lag_condition(s, r).astype(np.float32)

    # ---------------------------------------------------------------- helpers
    def _validate_engine_mode(self) -> None:
        if self.solver_config.engine in ("acoustic", "viscoacoustic") and self.config.mode not in _ACOUSTIC_MODES:
            raise ImagingError(f"acoustic/viscoacoustic engines image PP only, got imaging.mode={self.config.mode!r}")

    def _resolve_mode(self, mode: str | None = None) -> tuple[str, str]:
        m = str(mode if mode is not None else self.config.mode).lower()
        if m not in WAVE_MODES:
            raise ImagingError(f"unsupported imaging mode {m!r}")
        return WAVE_MODES[m]

    def _prepare_wavelet(self, shot: Any, spec: PropagationSpec, wavelet: np.ndarray | None) -> np.ndarray:
        if wavelet is not None:
            return np.ascontiguousarray(wavelet, dtype=np.float32)
        return source_wavelet(shot.source, spec.dt, spec.nt)

    def _prepare_record(self, shot: Any, spec: PropagationSpec, preprocess: Callable | None) -> dict[str, np.ndarray]:
        """imaging.py:396-423 — resample to spec.dt, optional hook, pad/trim to nt."""
        comps = dict(getattr(shot, "components", {}) or {})
        if not comps:
            comps["primary"] = shot.data
        out: dict[str, np.ndarray] = {}
        for name, arr in comps.items():
            data = np.asarray(arr)
            resample = abs(float(shot.dt) - spec.dt) > 1e-12 and data.shape[0] > 1
            if resample or preprocess is not None or data.dtype not in (np.float32, np.float64):
                # the reference works on a float64 copy; without resampling or a
                # hook the float32 samples pass unchanged (injection casts to float32)
                data = np.asarray(arr, dtype=np.float64)
            if resample:
                if preprocess is None:
                    # device sinc resampling: the record is cast to float32 for
                    # injection anyway, so one float32 rounding of the float64
                    # sums gives the reference's values
                    from .preprocess import resample_sinc as device_resample
                    data = np.asarray(device_resample(data, float(shot.dt), spec.dt), dtype=np.float64)
                else:
                    # the hook receives the float64 resampled record, as in the reference
                    data = num.resample_sinc(data, float(shot.dt), spec.dt)
            if preprocess is not None:
                data = np.asarray(preprocess(data, spec.dt), dtype=np.float64)
            out[name] = self._fit_length(data, int(spec.nt))
        return out

    @staticmethod
    def _fit_length(data: np.ndarray, nt: int) -> np.ndarray:
        if data.shape[0] >= nt:
            return data[:nt]
        padded = np.zeros((nt, data.shape[1]), dtype=data.dtype)
        padded[: data.shape[0]] = data
        return padded

    @staticmethod
    def _pml_mask(model: Any, spec: PropagationSpec) -> np.ndarray:
        nz, nx = model.shape
        n = int(spec.npml)
        mask = np.ones((nz, nx), dtype=np.float64)
        mask[:, :n] = 0.0
        mask[:, -n:] = 0.0
        mask[-n:, :] = 0.0
        if spec.boundary == "cpml":
            mask[:n, :] = 0.0
        return mask

    def _meta(self, spec, engine, shot, store, condition, start_step=0, prop=None, back=None, mode=None):
        q_meta: dict[str, Any] = {"model": str(self.q_config.model), "enabled": bool(self.q_config.enabled),
                                  "alpha_c": float(self.q_config.alpha_c), "f_ref": float(self.q_config.f_ref)}
        if engine == "viscoacoustic":
            fs = getattr(prop, "quality_summary", None)
            if isinstance(fs, dict):
                q_meta.update(fs)
            bs = getattr(back, "quality_summary", None)
            if isinstance(bs, dict):
                for key in ("compensation", "alpha_c", "alpha_mechanisms", "f_peak_mechanisms_hz", "f_max",
                            "gain_budget_db"):
                    if key in bs:
                        q_meta[key] = bs[key]
                q_meta["clipped_steps"] = int(bs.get("clipped", 0))
                q_meta["lowpass_steps"] = int(bs.get("lowpass_steps", 0))
        m = mode or self.config.mode
        a, b = self._resolve_mode(m)
        return {"placeholder": False, "method": "reverse-time migration (two-way wave equation)",
                "imager": self.name, "engine": engine, "condition": condition,
                "separation": self.config.separation, "modes": [f"{a}{b}"],
                "illumination": bool(self.config.illumination),
                "receiver_normalization": bool(self.config.receiver_normalization),
                "laplacian": bool(self.config.laplacian), "lowpass_fraction": float(self.config.lowpass_fraction),
                "checkpoints": store.summary(), "start_step": int(start_step),
                "start_periods": float(self.config.start_periods), "q": q_meta, "nt": int(spec.nt),
                "dt": float(spec.dt), "order": int(spec.order), "npml": int(spec.npml),
                "source_x": float(shot.source.x), "source_z": float(shot.source.z),
                "n_receivers": int(np.asarray(shot.receivers.x).size), "device": "B200 (sm_100a)",
                "accumulation": self.accumulation}


class ShotMigrator:
    """Device-resident RTM for one model: the forward and backward
    propagators are built once and reset between shots, so a stream of shots
    on the same model pays the material set-up once.  ``migrate`` returns
    ``ImageResult`` objects (host images); ``migrate_device`` takes the record
    as a device tensor and returns device tensors (torch, float32)."""

    def __init__(self, imager: RTMImager, model: Any) -> None:
        self.imager = imager
        self.model = model
        self.spec = PropagationSpec.from_config(imager.solver_config, model)
        try:
            check_stability(model, self.spec)
        except Exception as exc:
            raise ImagingError(str(exc)) from exc
        self.engine = imager.solver_config.engine
        self.prop = build_propagator(model, self.spec, engine=self.engine,
                                     q_options=imager.q_options(compensation=False))
        self.back = build_propagator(model, self.spec, engine=self.engine,
                                     q_options=imager.q_options(compensation=True))
        self._receivers_key: tuple | None = None
        self._used = False

    def interval_for(self, n_steps: int) -> int:
        """Checkpoint interval of a fresh run (state bytes before the first step)."""
        return checkpoint_interval(n_steps, max(int(self.prop.info().field_bytes), 1),
                                   float(self.imager.config.checkpoint_mb))

    def _prepare(self, source: Any, receivers: Any, modes: tuple[str, ...], n_steps: int):
        im = self.imager
        pairs = [im._resolve_mode(m) for m in modes]
        if not 1 <= len(pairs) <= 2:
            raise ImagingError("one or two imaging modes per pass")
        if self.engine in ("acoustic", "viscoacoustic") and any(m.lower() not in _ACOUSTIC_MODES for m in modes):
            raise ImagingError("acoustic/viscoacoustic engines image PP only; use solver.engine='elastic'")
        if self._used:
            self.prop.reset()
            self.back.reset()
        self._used = True
        self.prop.set_source(source)
        self.back.set_source(source)
        key = (np.asarray(receivers.x, dtype=np.float64).tobytes(), np.asarray(receivers.z, dtype=np.float64).tobytes())
        if key != self._receivers_key:
            self.prop.set_receivers(receivers)
            self.back.set_receivers(receivers)
            self._receivers_key = key
        else:
            self.prop._receivers = self.back._receivers = receivers
        per_state = max(int(self.prop.state_bytes()), 1)   # fields only before the first step
        interval = checkpoint_interval(n_steps, per_state, float(im.config.checkpoint_mb))
        store = CheckpointStore(interval=interval, bytes_per_state=per_state,
                                n_states=(n_steps + interval - 1) // interval)
        start_step = int(np.floor((float(source.delay) + float(im.config.start_periods)
                                   / max(float(source.f0), 1e-6)) / self.spec.dt))
        start_step = int(np.clip(start_step, 0, self.spec.nt))
        return pairs, store, start_step

    def _config(self, pairs, names, store, start_step, n_steps) -> _lib.MigrateConfig:
        im = self.imager
        condition = str(im.config.condition).lower()
        cfg = _lib.MigrateConfig()
        cfg.nt = int(n_steps)
        cfg.nt_spec = int(self.spec.nt)
        cfg.interval = int(store.interval)
        cfg.condition = _lib.COND[condition]
        # bit 0: source illumination (used only by normalized + illumination);
        # bit 1: receiver illumination (used only by receiver normalisation)
        cfg.illumination = (int(condition == "normalized" and bool(im.config.illumination))
                            | (2 if im.config.receiver_normalization else 0))
        cfg.start_step = start_step
        cfg.separation = _lib.SEP[im.config.separation]
        cfg.n_images = len(pairs)
        for k, (s, r) in enumerate(pairs):
            cfg.src_wave[k] = _lib.WAVE[s]
            cfg.rcv_wave[k] = _lib.WAVE[r]
        cfg.accum = _lib.ACCUM[im.accumulation]
        codes = [self.back._check_component(_target_component(n, self.engine), "inject") for n in names]
        if len(codes) > 8:
            raise ImagingError("at most 8 record components")
        cfg.n_comp = len(codes)
        for k, c in enumerate(codes):
            cfg.comp[k] = c
        return cfg

    def _post_args(self) -> dict:
        im = self.imager
        condition = str(im.config.condition).lower()
        g = self.model.grid
        return dict(dx=g.dx, dz=g.dz, by_illum=condition == "normalized" and bool(im.config.illumination),
                    by_rillum=bool(im.config.receiver_normalization), eps=float(im.config.eps),
                    laplacian=bool(im.config.laplacian), lowpass_fraction=float(im.config.lowpass_fraction),
                    npml=self.spec.npml, boundary=self.spec.boundary)

    def migrate(self, shot: Any, *, wavelet: np.ndarray | None = None, preprocess: Callable | None = None,
                modes: tuple[str, ...] = ("pp",)) -> list[ImageResult]:
        im = self.imager
        record = im._prepare_record(shot, self.spec, preprocess)
        if not record:
            raise ImagingError("empty shot record; nothing to back-propagate")
        w = im._prepare_wavelet(shot, self.spec, wavelet)
        pairs, store, start_step = self._prepare(shot.source, shot.receivers, modes, len(w))
        names = list(record)
        cfg = self._config(pairs, names, store, start_step, len(w))
        rec = np.ascontiguousarray(np.stack([np.asarray(record[n], dtype=np.float32) for n in names]))
        g = self.model.grid
        acc = np.zeros((3, len(pairs), g.nz, g.nx))
        _lib.check(_lib.lib().ertm_migrate(self.prop.handle, self.back.handle, cfg, _lib.ptr(w), _lib.ptr(rec),
                                          _lib.ptr(acc[0]), _lib.ptr(acc[1]), _lib.ptr(acc[2])), "migrate")
        self.prop._psi_allocated = self.back._psi_allocated = True
        condition = str(im.config.condition).lower()
        results = []
        for k, m in enumerate(modes):
            image = postprocess_image(acc[0, k], acc[1, k], acc[2, k], **self._post_args())
            res = ImageResult(image=image, grid=g, mode=m,
                              meta=im._meta(self.spec, self.engine, shot, store, condition, start_step, self.prop,
                                            self.back, m))
            res.validate()
            results.append(res)
        return results

    def migrate_device(self, source: Any, receivers: Any, record, names: list[str], wavelet: np.ndarray, *,
                       modes: tuple[str, ...] = ("pp",), stream: int | None = None):
        """Device-resident form: ``record`` is a contiguous device tensor
        (n_comp, nt, nrec) float32 already aligned to the propagation dt;
        returns a device tensor (n_modes, nz, nx) float32 of final images."""
        import torch

        w = np.ascontiguousarray(wavelet, dtype=np.float32)
        pairs, store, start_step = self._prepare(source, receivers, modes, len(w))
        cfg = self._config(pairs, names, store, start_step, len(w))
        g = self.model.grid
        dev = record.device
        acc = torch.empty((3, len(pairs), g.nz, g.nx), dtype=torch.float64, device=dev)
        _lib.check(_lib.lib().ertm_migrate(self.prop.handle, self.back.handle, cfg, _lib.ptr(w), _lib.ptr(record),
                                          _lib.ptr(acc[0]), _lib.ptr(acc[1]), _lib.ptr(acc[2])), "migrate")
        self.prop._psi_allocated = self.back._psi_allocated = True
        out = torch.empty((len(pairs), g.nz, g.nx), dtype=torch.float32, device=dev)
        a = self._post_args()
        for k in range(len(pairs)):
            _lib.check(_lib.lib().ertm_postprocess(
                g.nz, g.nx, float(a["dx"]), float(a["dz"]), _lib.ptr(acc[0, k]), _lib.ptr(acc[1, k]),
                _lib.ptr(acc[2, k]), int(a["by_illum"]), int(a["by_rillum"]), a["eps"], int(a["laplacian"]),
                a["lowpass_fraction"], int(a["npml"]), int(a["boundary"] == "cpml"), _lib.ptr(out[k]), stream),
                "postprocess")
        return out


def pair_device_bytes(mig: ShotMigrator) -> int:
    """Device memory a migrator's two propagators hold between runs: state
    fields and (an upper bound on) the coefficient block, twice."""
    info = mig.prop.info()
    return 2 * (int(info.state_bytes) + 12 * info.nzp * info.ld * 4)


class MigratorPool:
    """Propagator pairs kept between calls, per model object.

    Building a ``ShotMigrator`` uploads the model, derives the CPML profiles
    and (viscoacoustic) fits the relaxation tables; a stream of calls on one
    model pays that once.  ``begin`` starts a call: it frees the pairs of
    models the call does not use, pairs beyond the call's shot count of a
    model, and pairs whose inputs changed since they were built (the imager's
    solver or Q settings, the grid, or the material arrays changed in place).
    ``take`` hands out a model's pairs in order within one group of shots
    and builds another only when the group holds more shots of that model
    than any group before."""

    _FIELDS = ("vp", "vs", "rho", "qp", "qs")

    def __init__(self, imager: "RTMImager") -> None:
        # a weak reference: an imager that owns its pool is freed, with the
        # pool's device memory, as soon as the last reference to it goes
        self._imager = weakref.ref(imager)
        # id(model) -> (model, the inputs its pairs were built from, pairs)
        self._entries: dict[int, tuple[Any, tuple, list[ShotMigrator]]] = {}

    @property
    def imager(self) -> "RTMImager":
        im = self._imager()
        if im is None:
            raise ImagingError("the imager of this migrator pool no longer exists")
        return im

    def _inputs(self, model: Any) -> tuple:
        im = self.imager
        g = model.grid
        arrays = tuple(None if getattr(model, n, None) is None else np.array(getattr(model, n), copy=True)
                       for n in self._FIELDS)
        settings = (repr(im.solver_config), repr(im.q_options(compensation=False)),
                    repr(im.q_options(compensation=True)),
                    tuple(getattr(g, a, None) for a in ("nx", "nz", "dx", "dz", "x0", "z0")))
        return settings, arrays

    @staticmethod
    def _same(a: tuple, b: tuple) -> bool:
        if a[0] != b[0]:
            return False
        for x, y in zip(a[1], b[1]):
            if (x is None) != (y is None):
                return False
            if x is not None and (x.shape != y.shape or not np.array_equal(x, y)):
                return False
        return True

    def begin(self, models: list) -> None:
        counts: dict[int, int] = {}
        for m in models:
            counts[id(m)] = counts.get(id(m), 0) + 1
        for key in list(self._entries):
            model, inputs, migs = self._entries[key]
            # a live pooled model and a model of this call with the same id
            # are the same object (the pool holds a reference to it)
            if key not in counts or not self._same(inputs, self._inputs(model)):
                del self._entries[key]
            else:
                del migs[counts[key]:]

    def take(self, model: Any, taken: dict[int, int]) -> ShotMigrator:
        key = id(model)
        entry = self._entries.get(key)
        if entry is None:
            entry = self._entries[key] = (model, self._inputs(model), [])
        k = taken.get(key, 0)
        taken[key] = k + 1
        if k == len(entry[2]):
            entry[2].append(ShotMigrator(self.imager, model))
        return entry[2][k]

    def sizer(self, model: Any) -> ShotMigrator:
        """A pair of ``model`` to size a shot with (every pair of a model has
        the same footprint), built if the model has none yet; it is not
        taken."""
        return self.take(model, {})

    def held_bytes(self) -> int:
        return sum(pair_device_bytes(m) for _, _, migs in self._entries.values() for m in migs)

    def clear(self) -> None:
        """Drop every pair (their device memory is freed)."""
        self._entries.clear()


def build_imager(config: ImagingConfig, solver_config: SolverConfig | None = None,
                 q_config: QConfig | None = None) -> RTMImager:
    return RTMImager(config, solver_config, q_config)


__all__ = ["WAVE_MODES", "zero_lag_condition", "normalized_terms", "excitation_terms", "CheckpointStore",
           "checkpoint_interval", "record_source_wavefield", "replay_block", "postprocess_image", "RTMImager",
           "ShotMigrator", "build_imager", "SolverError"]
