"""Record preprocessing on the device (preprocess.py:36-224 of the reference).

Same functions, signatures and results as the reference's ``ertm.preprocess``
(rotation of the horizontal components, sinc resampling to a new ``dt``,
direct-wave mute, end taper, and ``prepare_shot`` chaining them), with the
per-sample work on the GPU: ``ertm_rotate``, ``ertm_resample``, ``ertm_mute``
and ``ertm_taper`` compute in float64 and round to float32 once, as the
reference does.  Only O(nt) or O(nrec) set-up (the resampling weights, the
mute times, the taper ramp) is evaluated on the host, with the reference's
formulas.
"""

from __future__ import annotations

from dataclasses import replace
from typing import Sequence

import numpy as np

from . import _lib
from .exceptions import DataError

_MIN_SAMPLES = 3


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _as_2d(a: np.ndarray) -> tuple[np.ndarray, bool]:
    a = _f32(a)
    if a.ndim == 1:
        return a[:, None].copy(), True
    if a.ndim != 2:
        raise DataError(f"only 1-D/2-D records, got {a.ndim}-D")
    return a, False


# ---------------------------------------------------------------------------
# rotation (preprocess.py:36-83)
# ---------------------------------------------------------------------------
def rotate_components(components: dict[str, np.ndarray], angle_deg: float) -> dict[str, np.ndarray]:
    """vx' = cos·vx + sin·vz, vz' = −sin·vx + cos·vz; p unchanged."""
    if not components:
        raise DataError("rotation needs at least one component")
    angle = np.deg2rad(float(angle_deg))
    cos, sin = float(np.cos(angle)), float(np.sin(angle))
    rotated = {name: np.array(array, copy=True) for name, array in components.items()}
    if "vx" in components and "vz" in components:
        vx, vz = _f32(components["vx"]), _f32(components["vz"])
        if vx.shape != vz.shape:
            raise DataError("vx and vz differ in shape")
        ox, oz = np.empty_like(vx), np.empty_like(vz)
        _lib.check(_lib.lib().ertm_rotate(_lib.ptr(vx), _lib.ptr(vz), vx.size, cos, sin, _lib.ptr(ox), _lib.ptr(oz),
                                         None), "rotate")
        rotated["vx"], rotated["vz"] = ox, oz
    return rotated


def rotate_shot(shot, angle_deg: float):
    if angle_deg == 0.0:
        return shot
    components = rotate_components(shot.components, angle_deg)
    primary_name = "p" if "p" in components else ("vz" if "vz" in components else None)
    data = components[primary_name] if primary_name else shot.data
    return replace(shot, data=data, components=components, meta={**shot.meta, "rotation_deg": angle_deg})


# ---------------------------------------------------------------------------
# sinc resampling (numerics.py:337-392, preprocess.py:89-121)
# ---------------------------------------------------------------------------
def resample_weights(n_in: int, dt_in: float, dt_out: float, half_length: int = 8,
                     beta: float = 8.6) -> tuple[np.ndarray, np.ndarray]:
    """Kaiser-windowed sinc weights (n_out × 2·half_length, normalised per
    output sample) and the first tap offset of each output sample."""
    if dt_in <= 0 or dt_out <= 0:
        raise ValueError("dt_in / dt_out must be positive")
    if n_in < _MIN_SAMPLES:
        raise ValueError(f"too few samples ({n_in}) to interpolate")
    n_out = int(np.floor((n_in - 1) * dt_in / dt_out + 1e-9)) + 1
    pos = np.arange(n_out, dtype=np.float64) * (dt_out / dt_in)
    taps = np.arange(-half_length + 1, half_length + 1)
    base = np.floor(pos).astype(np.int64)
    off = base[:, None] + taps[None, :]
    w = np.sinc(pos[:, None] - off) * np.kaiser(2 * half_length, beta)[None, :]
    s = w.sum(axis=1, keepdims=True)
    s[s == 0] = 1.0
    w /= s
    return np.ascontiguousarray(w), np.ascontiguousarray(base - half_length + 1)


def resample_sinc(data: np.ndarray, dt_in: float, dt_out: float, *, axis: int = 0, half_length: int = 8,
                  beta: float = 8.6) -> np.ndarray:
    """The reference's numerics.resample_sinc on the device; float32 result
    (the reference's float64 result rounded once)."""
    a = np.asarray(data)
    if axis == 1:
        a = a.T
    arr, squeeze = _as_2d(a)
    w, off0 = resample_weights(arr.shape[0], dt_in, dt_out, half_length, beta)
    n_out = w.shape[0]
    out = np.empty((n_out, arr.shape[1]), dtype=np.float32)
    _lib.check(_lib.lib().ertm_resample(_lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(w), _lib.ptr(off0),
                                       w.shape[1], n_out, _lib.ptr(out), None), "resample")
    if squeeze:
        out = out[:, 0]
    return out.T.copy() if axis == 1 else out


def resample_shot(shot, dt_target: float):
    if abs(dt_target - shot.dt) < 1e-12:
        return shot
    if dt_target <= 0:
        raise DataError(f"dt_target must be positive, got {dt_target}")
    components = dict(shot.components) or {"primary": shot.data}
    converted = {name: resample_sinc(array, shot.dt, dt_target) for name, array in components.items()}
    primary = "primary" if "primary" in converted else next(iter(converted))
    nt = converted[primary].shape[0]
    t = np.arange(nt, dtype=np.float64) * dt_target
    data = converted[primary]
    new_components = {} if "primary" in converted else dict(converted)
    return replace(shot, data=data, dt=float(dt_target), t=t, components=new_components,
                   meta={**shot.meta, "input_dt": float(shot.dt), "resampled_dt": float(dt_target),
                         "resampled": True})


def required_dt(model, dx: float | None = None, *, order: int = 8) -> float:
    from .numerics import cfl_dt
    dx = model.grid.dx if dx is None else dx
    return cfl_dt(float(np.max(model.vp)), dx, model.grid.dz, order, safety=0.5)


# ---------------------------------------------------------------------------
# direct-wave mute and end taper (preprocess.py:121-191)
# ---------------------------------------------------------------------------
def _mute(array: np.ndarray, t: np.ndarray, start: np.ndarray, end: np.ndarray) -> np.ndarray:
    a, squeeze = _as_2d(array)
    out = np.empty_like(a)
    _lib.check(_lib.lib().ertm_mute(_lib.ptr(a), a.shape[0], a.shape[1], _lib.ptr(t), _lib.ptr(start), _lib.ptr(end),
                                   _lib.ptr(out), None), "mute")
    return out[:, 0] if squeeze else out


def mute_direct_wave(shot, v_reference: float, *, margin_periods: float = 1.2, offset_factor: float = 1.05,
                     taper_periods: float = 0.5):
    """t_mute(x) = delay + margin/f0 + offset_factor·|x − x_s|/v_ref with a
    cosine ramp of ±taper_periods/f0 around it."""
    if v_reference <= 0:
        raise DataError(f"v_reference must be positive, got {v_reference}")
    t = np.ascontiguousarray(np.asarray(shot.t, dtype=np.float64))
    offset = np.abs(np.asarray(shot.receivers.x, dtype=np.float64) - shot.source.x)
    period = 1.0 / max(float(shot.source.f0), 1e-6)
    t_mute = float(shot.source.delay) + margin_periods * period + offset_factor * offset / v_reference
    taper = max(float(taper_periods) * period, 1e-9)
    start = np.ascontiguousarray(t_mute - taper)
    end = np.ascontiguousarray(t_mute + taper)
    data = _mute(shot.data, t, start, end)
    components = {name: _mute(array, t, start, end) for name, array in shot.components.items()}
    primary = components.get("p", data) if components else data
    return replace(shot, data=primary, components=components,
                   meta={**shot.meta, "direct_mute": True, "mute_velocity": float(v_reference)})


def _taper(array: np.ndarray, fraction: float) -> np.ndarray:
    a, squeeze = _as_2d(array)
    n = a.shape[0]
    w = max(int(fraction * n), 1)
    ramp = np.ascontiguousarray(0.5 - 0.5 * np.cos(np.pi * (np.arange(w) + 0.5) / w))
    out = np.empty_like(a)
    _lib.check(_lib.lib().ertm_taper(_lib.ptr(a), n, a.shape[1], _lib.ptr(ramp), w, _lib.ptr(out), None), "taper")
    return out[:, 0] if squeeze else out


def taper_record_ends(shot, fraction: float = 0.05):
    if not 0 < fraction < 0.5:
        raise DataError(f"fraction must lie in (0, 0.5), got {fraction}")
    data = _taper(shot.data, fraction)
    components = {name: _taper(array, fraction) for name, array in shot.components.items()}
    primary = components.get("p", data) if components else data
    return replace(shot, data=primary, components=components, meta={**shot.meta, "taper_fraction": fraction})


def prepare_shot(shot, *, model, record_dt: float | None = None, rotation_deg: float = 0.0, mute: bool = True,
                 v_reference: float | None = None, taper_fraction: float = 0.05):
    """Rotation → resampling → direct-wave mute → end taper (preprocess.py:194-224)."""
    prepared = shot
    if rotation_deg:
        prepared = rotate_shot(prepared, rotation_deg)
    if record_dt is not None and abs(record_dt - prepared.dt) > 1e-12:
        prepared = resample_shot(prepared, record_dt)
    if mute:
        velocity = float(v_reference) if v_reference is not None else float(np.percentile(model.vp, 25))
        prepared = mute_direct_wave(prepared, velocity)
    if taper_fraction > 0:
        prepared = taper_record_ends(prepared, taper_fraction)
    return prepared


def build_shot_sequence(base_shot, source_positions: Sequence[float]) -> list:
    return [replace(base_shot, source=replace(base_shot.source, x=float(x)), meta={**base_shot.meta, "shot_x": float(x)})
            for x in source_positions]
