"""Data-domain Q filtering on the device (qcomp.py of the reference).

``time_varying_filter`` is the reference's short-time Fourier overlap-add
filter with the framing, FFTs, per-frame responses and overlap-add on the GPU
(``ertm_stft_filter``, cuFFT double); the per-frame responses — one complex
vector of L/2+1 frequencies per frame, from the caller's ``response_fn`` —
are evaluated on the host as in the reference.  ``QCompensator`` is the
``preprocess=`` hook of ``RTMImager.migrate`` in the reference's filter mode.
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


def q_response(freqs: np.ndarray, travel_time: float, q: float, f_ref: float, *, strength: float = 1.0,
               amplitude: bool = True, dispersion: bool = True) -> np.ndarray:
    """Constant-Q response exp(−π f t*/Q)·exp(iφ), φ = −(2 f t*/Q)·ln(f/f_ref) (qcomp.py:44-62)."""
    if q <= 0:
        raise DataError(f"Q must be positive, got {q}")
    f = np.abs(np.asarray(freqs, dtype=np.float64))
    f_safe = np.where(f > 1e-9, f, 1e-9)
    t_star = float(travel_time) * float(strength)
    response = np.ones_like(f, dtype=np.complex128)
    if amplitude:
        response *= np.exp(-np.pi * f * t_star / float(q))
    if dispersion:
        phase = -2.0 * f * t_star / float(q) * np.log(f_safe / float(f_ref))
        response *= np.exp(1j * phase)
    return response


def compensation_response(freqs: np.ndarray, travel_time: float, q: float, f_ref: float, *, alpha_c: float = 0.8,
                          gain_cap: float = 30.0, lowpass: np.ndarray | None = None) -> np.ndarray:
    """Inverse-Q gain (exponent scaled by α_c, capped) with the opposite phase (qcomp.py:65-87)."""
    if not 0.0 <= alpha_c <= 1.0:
        raise DataError(f"alpha_c must lie in [0, 1], got {alpha_c}")
    f = np.abs(np.asarray(freqs, dtype=np.float64))
    f_safe = np.where(f > 1e-9, f, 1e-9)
    t_star = float(travel_time) * float(alpha_c)
    gain = np.minimum(np.exp(np.pi * f * t_star / float(q)), float(gain_cap))
    phase = 2.0 * f * t_star / float(q) * np.log(f_safe / float(f_ref))
    response = gain * np.exp(1j * phase)
    if lowpass is not None:
        response = response * np.asarray(lowpass, dtype=np.float64)
    return response


def time_varying_filter(data: np.ndarray, dt: float, response_fn: Callable[[float, np.ndarray], np.ndarray], *,
                        nperseg: int = 128, overlap: float = 0.5) -> np.ndarray:
    """Overlap-add filtering with one response per frame (qcomp.py:98-147); float64 result."""
    array = np.asarray(data, dtype=np.float64)
    if array.ndim == 1:
        array, squeeze = array[:, None], True
    elif array.ndim == 2:
        squeeze = False
    else:
        raise DataError(f"only 1-D/2-D data, got {array.ndim}-D")
    if dt <= 0:
        raise DataError(f"dt must be positive, got {dt}")
    n = array.shape[0]
    L = int(min(max(nperseg, 8), max(n, 8)))
    hop = max(int(L * (1.0 - overlap)), 1)
    window = np.ascontiguousarray(np.hanning(L))
    freqs = np.fft.rfftfreq(L, d=dt)
    responses = []
    for start in range(0, n, hop):
        if min(start + L, n) - start < 4:
            break
        r = np.asarray(response_fn((start + 0.5 * L) * dt, freqs), dtype=np.complex128)
        if r.shape[0] != freqs.size:
            raise DataError(f"response has {r.shape[0]} points, the frame spectrum {freqs.size}")
        responses.append(r)
    out = np.zeros_like(array)
    if responses:
        resp = np.ascontiguousarray(np.stack(responses))
        src = np.ascontiguousarray(array)
        _lib.check(_lib.lib().ertm_stft_filter(_lib.ptr(src), n, array.shape[1], L, hop, len(responses),
                                              _lib.ptr(window), _lib.ptr(resp.view(np.float64)), _lib.ptr(out),
                                              None), "stft filter")
    return out[:, 0] if squeeze else out


def attenuate_record(data: np.ndarray, dt: float, q: float, *, f_ref: float = 30.0, strength: float = 1.0,
                     nperseg: int = 128) -> np.ndarray:
    """Constant-Q attenuation and dispersion of a record (qcomp.py:150-168)."""
    return time_varying_filter(data, dt, lambda tc, f: q_response(f, max(tc, 1e-6), q, f_ref, strength=strength),
                               nperseg=nperseg)


@dataclass
class QCompensator:
    """Receiver-side Q compensation, usable as ``migrate(preprocess=...)`` (qcomp.py:171-213)."""

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
        q, alpha, cap = float(self.q_value), float(self.config.alpha_c), float(self.config.gain_cap)
        f_ref = float(self.config.f_ref)
        nyquist = 0.5 / dt

        def response(t_center: float, freqs: np.ndarray) -> np.ndarray:
            travel = max(t_center, 1e-6)
            cutoff_ratio = 0.95 - 0.35 * min(travel / 0.5, 1.0)
            cutoff = max(nyquist * cutoff_ratio, 2.0 * f_ref)
            lowpass = 1.0 / (1.0 + (np.abs(freqs) / cutoff) ** 4)
            return compensation_response(freqs, travel, q, f_ref, alpha_c=alpha, gain_cap=cap, lowpass=lowpass)

        return time_varying_filter(data, dt, response, nperseg=self.nperseg)


def build_compensator(config: QConfig, model_qp: float, model_qs: float, *, wave: str = "P") -> QCompensator:
    q_value = float(model_qp if str(wave).upper().startswith("P") else model_qs)
    return QCompensator(config=config, q_value=q_value, wave=str(wave))
