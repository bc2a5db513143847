"""Data-domain Q filtering on the device (the reference's qcomp.py).

The filter is a short-time Fourier overlap-add: a record is cut into
Hann-windowed frames, every frame's spectrum is multiplied by a response
that depends on the frame's centre time, and the frames are added back.  The
framing, transforms, multiplication and overlap-add of all frames of all
traces run in one device call (``ertm_stft_filter``).

Responses are built here as one complex table of shape (frames, L/2+1)
per record, with NumPy broadcasting over frame times and frequencies:

* attenuation (the forward constant-Q model, qcomp.py:44-62)
  log-amplitude −π f t*/Q, phase −(2 f t*/Q)·ln(f/f_ref), t* = strength·t;
* compensation (its regularised inverse, qcomp.py:65-87, 171-198)
  amplitude min(exp(π f α t/Q), cap), phase +(2 f α t/Q)·ln(f/f_ref), times a
  4th-order low-pass 1/(1 + (f/f_c)^4) whose corner f_c(t) =
  max(ν·(0.95 − 0.35·min(t/0.5, 1)), 2 f_ref) falls with time (ν the Nyquist
  frequency).

These are the reference's physical formulas (the outputs must agree);
frequencies below 1e-9 Hz use 1e-9 in the logarithm as the reference does.
``q_response``, ``compensation_response`` and ``time_varying_filter`` keep
the reference's names and signatures for callers that use them directly.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np

from . import _lib
from .config import QConfig
from .exceptions import DataError

__all__ = ["DataError", "QCompensator", "attenuate_record", "build_compensator", "compensation_response",
           "q_response", "time_varying_filter"]

_F_FLOOR = 1e-9     # frequencies in the logarithm are floored here (0 Hz has no dispersion)


# ---------------------------------------------------------------------------
# response tables: rows = frame centre times, columns = frequencies
# ---------------------------------------------------------------------------
def _grid(freqs: np.ndarray, times) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    f = np.abs(np.asarray(freqs, dtype=np.float64))[None, :]
    t = np.asarray(times, dtype=np.float64).reshape(-1, 1)
    log_ratio_floor = np.where(f > _F_FLOOR, f, _F_FLOOR)
    return f, t, log_ratio_floor


def _attenuation_table(freqs: np.ndarray, times, q: float, f_ref: float, strength: float = 1.0,
                       amplitude: bool = True, dispersion: bool = True) -> np.ndarray:
    """(frames, freqs) constant-Q responses for travel times ``times``."""
    if q <= 0:
        raise DataError(f"Q must be positive, got {q}")
    f, t, ff = _grid(freqs, times)
    decay = f * (t * float(strength)) / float(q)          # f·t*/Q
    table = np.ones(np.broadcast_shapes(f.shape, t.shape), dtype=np.complex128)
    if amplitude:
        table *= np.exp(-np.pi * decay)
    if dispersion:
        table *= np.exp(1j * (-2.0 * decay * np.log(ff / float(f_ref))))
    return table


def _compensation_table(freqs: np.ndarray, times, q: float, f_ref: float, alpha_c: float, gain_cap: float,
                        corner=None) -> np.ndarray:
    """(frames, freqs) inverse-Q responses; ``corner`` (per frame, Hz) adds
    the 4th-order low-pass."""
    if not 0.0 <= alpha_c <= 1.0:
        raise DataError(f"alpha_c must lie in [0, 1], got {alpha_c}")
    f, t, ff = _grid(freqs, times)
    growth = f * (t * float(alpha_c)) / float(q)          # f·α·t/Q
    gain = np.minimum(np.exp(np.pi * growth), float(gain_cap))
    table = gain * np.exp(1j * (2.0 * growth * np.log(ff / float(f_ref))))
    if corner is not None:
        fc = np.asarray(corner, dtype=np.float64).reshape(-1, 1)
        table = table * (1.0 / (1.0 + (f / fc) ** 4))
    return table


def q_response(freqs: np.ndarray, travel_time: float, q: float, f_ref: float, *, strength: float = 1.0,
               amplitude: bool = True, dispersion: bool = True) -> np.ndarray:
    """Constant-Q response at one travel time (qcomp.py:44-62)."""
    return _attenuation_table(freqs, [travel_time], q, f_ref, strength, amplitude, dispersion)[0]


def compensation_response(freqs: np.ndarray, travel_time: float, q: float, f_ref: float, *, alpha_c: float = 0.8,
                          gain_cap: float = 30.0, lowpass: np.ndarray | None = None) -> np.ndarray:
    """Inverse-Q response at one travel time, optionally times a real
    per-frequency ``lowpass`` (qcomp.py:65-87)."""
    row = _compensation_table(freqs, [travel_time], q, f_ref, alpha_c, gain_cap)[0]
    return row if lowpass is None else row * np.asarray(lowpass, dtype=np.float64)


# ---------------------------------------------------------------------------
# the filter
# ---------------------------------------------------------------------------
@dataclass
class _Frames:
    length: int          # samples per frame
    hop: int
    centres: np.ndarray  # frame centre times (s), frames with at least 4 samples
    freqs: np.ndarray    # rfft frequencies of a frame (Hz)


def _frames(n: int, dt: float, nperseg: int, overlap: float) -> _Frames:
    """Frame layout of qcomp.py:98-147: length clipped to [8, max(n, 8)],
    hop L·(1 − overlap), frames until fewer than 4 samples remain."""
    if dt <= 0:
        raise DataError(f"dt must be positive, got {dt}")
    length = int(min(max(nperseg, 8), max(n, 8)))
    hop = max(int(length * (1.0 - overlap)), 1)
    starts = np.arange(0, n, hop)
    starts = starts[np.minimum(starts + length, n) - starts >= 4]
    return _Frames(length, hop, (starts + 0.5 * length) * dt, np.fft.rfftfreq(length, d=dt))


def _as_traces(data: np.ndarray) -> tuple[np.ndarray, bool]:
    a = np.asarray(data, dtype=np.float64)
    if a.ndim == 1:
        return a[:, None], True
    if a.ndim != 2:
        raise DataError(f"only 1-D/2-D data, got {a.ndim}-D")
    return a, False


def _apply(traces: np.ndarray, fr: _Frames, table: np.ndarray) -> np.ndarray:
    """Run the device overlap-add with one response row per frame."""
    out = np.zeros_like(traces)
    if len(fr.centres):
        if table.shape != (len(fr.centres), fr.freqs.size):
            raise DataError(f"response table {table.shape}, frames x frequencies "
                            f"{(len(fr.centres), fr.freqs.size)}")
        resp = np.ascontiguousarray(table, dtype=np.complex128)
        src = np.ascontiguousarray(traces)
        window = np.ascontiguousarray(np.hanning(fr.length))
        _lib.check(_lib.lib().ertm_stft_filter(_lib.ptr(src), traces.shape[0], traces.shape[1], fr.length, fr.hop,
                                              len(fr.centres), _lib.ptr(window), _lib.ptr(resp.view(np.float64)),
                                              _lib.ptr(out), None), "stft filter")
    return out


def time_varying_filter(data: np.ndarray, dt: float, response_fn: Callable[[float, np.ndarray], np.ndarray], *,
                        nperseg: int = 128, overlap: float = 0.5) -> np.ndarray:
    """Overlap-add filtering with ``response_fn(centre_time, freqs)`` per
    frame (qcomp.py:98-147); float64 result of the input's shape."""
    traces, squeeze = _as_traces(data)
    fr = _frames(traces.shape[0], dt, nperseg, overlap)
    rows = [np.asarray(response_fn(float(tc), fr.freqs), dtype=np.complex128) for tc in fr.centres]
    for r in rows:
        if r.shape != fr.freqs.shape:
            raise DataError(f"response has {r.shape[0]} points, the frame spectrum {fr.freqs.size}")
    out = _apply(traces, fr, np.stack(rows) if rows else np.zeros((0, fr.freqs.size), np.complex128))
    return out[:, 0] if squeeze else out


def attenuate_record(data: np.ndarray, dt: float, q: float, *, f_ref: float = 30.0, strength: float = 1.0,
                     nperseg: int = 128) -> np.ndarray:
    """Constant-Q attenuation and dispersion of a record (qcomp.py:150-168)."""
    if q <= 0:
        raise DataError(f"Q must be positive, got {q}")
    traces, squeeze = _as_traces(data)
    fr = _frames(traces.shape[0], dt, nperseg, 0.5)
    table = _attenuation_table(fr.freqs, np.maximum(fr.centres, 1e-6), q, f_ref, strength)
    out = _apply(traces, fr, table)
    return out[:, 0] if squeeze else out


@dataclass
class QCompensator:
    """Receiver-side Q compensation, usable as ``migrate(preprocess=...)``
    (qcomp.py:171-213): inverse-Q gain and phase with a low-pass whose
    corner falls with the frame's travel time."""

    config: QConfig
    q_value: float = 100.0
    wave: str = "P"
    nperseg: int = 128

    def __post_init__(self) -> None:
        self.config.validate()
        if self.q_value <= 0:
            raise DataError(f"q_value must be positive, got {self.q_value}")

    def __call__(self, data: np.ndarray, dt: float) -> np.ndarray:
        if not self.config.enabled:
            return np.asarray(data)
        traces, squeeze = _as_traces(data)
        fr = _frames(traces.shape[0], dt, self.nperseg, 0.5)
        travel = np.maximum(fr.centres, 1e-6)
        f_ref = float(self.config.f_ref)
        corner = np.maximum((0.5 / dt) * (0.95 - 0.35 * np.minimum(travel / 0.5, 1.0)), 2.0 * f_ref)
        table = _compensation_table(fr.freqs, travel, float(self.q_value), f_ref, float(self.config.alpha_c),
                                    float(self.config.gain_cap), corner)
        out = _apply(traces, fr, table)
        return out[:, 0] if squeeze else out


def build_compensator(config: QConfig, model_qp: float, model_qs: float, *, wave: str = "P") -> QCompensator:
    """The compensator for the P (qp) or S (qs) wave's Q."""
    q_value = float(model_qp if str(wave).upper().startswith("P") else model_qs)
    return QCompensator(config=config, q_value=q_value, wave=str(wave))
