"""GSLS constant-Q fit and relaxation tables (host, float64).

Set-up for the viscoacoustic engine: the per-Q least-squares fit of the
relaxation times τ_l and strengths Δ_l (viscoelastic.py:132-205), the
compensation regularisation (propagation.py:607-639), and the small per-Q
tables the CUDA kernels index.  The per-cell coefficient expansion
(K_R, b_l) happens on the device.
"""

from __future__ import annotations

import copy
import threading

from dataclasses import dataclass, field
from typing import Iterable

import numpy as np

from .exceptions import ERTMError


def normalized_modulus(tau_sigma: Iterable[float], delta: Iterable[float], freqs: Iterable[float]) -> np.ndarray:
    """K(ω)/K_R = 1 − Σ Δ_l / (1 + iωτ_l)."""
    omega = 2.0 * np.pi * np.asarray(freqs, dtype=np.float64)
    out = np.ones_like(omega, dtype=np.complex128)
    for tau, dlt in zip(tau_sigma, delta):
        out -= dlt / (1.0 + 1j * omega * tau)
    return out


@dataclass(frozen=True)
class GSLSParameters:
    q: float
    f_ref: float
    tau_sigma: tuple[float, ...]
    delta: tuple[float, ...]
    k_relaxed: float
    k_unrelaxed: float
    f_band: tuple[float, float] = (0.0, 0.0)
    fit_error: float = 0.0

    def modulus(self, freqs: Iterable[float]) -> np.ndarray:
        return normalized_modulus(self.tau_sigma, self.delta, freqs)

    def quality(self, freqs: Iterable[float]) -> np.ndarray:
        m = self.modulus(freqs)
        re, im = np.real(m), np.imag(m)
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.where(np.abs(im) > 1e-12, re / im, np.inf)

    def phase_velocity(self, freqs: Iterable[float], vp: float) -> np.ndarray:
        mod = np.real(self.modulus(freqs))
        ref = float(np.real(self.modulus([self.f_ref])[0]))
        return vp * np.sqrt(np.maximum(mod, 1e-9) / max(ref, 1e-12))


def _pack(q, f_ref, tau, delta, band, error) -> GSLSParameters:
    return GSLSParameters(q=float(q), f_ref=float(f_ref), tau_sigma=tuple(float(t) for t in tau),
                          delta=tuple(float(d) for d in delta), k_relaxed=1.0,
                          k_unrelaxed=float(1.0 + np.sum(delta)), f_band=(float(band[0]), float(band[1])),
                          fit_error=float(error))


def _single_mechanism(q: float, f_ref: float) -> tuple[float, float]:
    """Analytic one-mechanism fit with its Q minimum at f_ref."""
    u = (-1.0 + np.sqrt(1.0 + q * q)) / max(q, 1e-12)
    return float(u / (2.0 * np.pi * f_ref)), float(1.0 - u * u)


_FIT_CACHE: dict[tuple, GSLSParameters] = {}
_FIT_LOCK = threading.Lock()


def fit_gsls(q: float, f_ref: float, *, n_mechanisms: int = 3, band_ratio: float = 1.5,
             min_q: float = 2.0) -> GSLSParameters:
    """Least-squares constant-Q fit over [f_ref/band, f_ref·band] in log Q.

    The fit is a pure function of its arguments and takes ~0.1 s, so results
    are memoised per process (a copy is returned each time)."""
    key = (float(q), float(f_ref), int(n_mechanisms), float(band_ratio), float(min_q))
    with _FIT_LOCK:
        hit = _FIT_CACHE.get(key)
    if hit is None:
        hit = _fit_gsls(*key)
        with _FIT_LOCK:
            _FIT_CACHE[key] = hit
    return copy.deepcopy(hit)


def _fit_gsls(q: float, f_ref: float, n_mechanisms: int, band_ratio: float, min_q: float) -> GSLSParameters:
    if q <= min_q:
        raise ERTMError(f"GSLS fit needs Q > {min_q}, got {q}")
    if f_ref <= 0:
        raise ERTMError(f"f_ref must be positive, got {f_ref}")
    f_lo, f_hi = f_ref / band_ratio, f_ref * band_ratio
    freqs = np.geomspace(f_lo, f_hi, 24)
    if q > 1.0e4 or int(n_mechanisms) <= 1:
        tau, dlt = _single_mechanism(q, f_ref)
        return _pack(q, f_ref, [tau], [dlt], (f_lo, f_hi), 0.0)
    from scipy.optimize import least_squares

    n = int(n_mechanisms)
    tau0 = 1.0 / (2.0 * np.pi * np.geomspace(f_lo, f_hi, n))
    delta0 = np.full(n, 2.0 / q)
    weights = 1.0 + 0.5 * np.exp(-0.5 * (np.log(freqs / f_ref) / 0.25) ** 2)

    def residual(p: np.ndarray) -> np.ndarray:
        m = normalized_modulus(tuple(np.exp(p[:n])), tuple(np.exp(p[n:])), freqs)
        re, im = np.real(m), np.imag(m)
        with np.errstate(divide="ignore", invalid="ignore"):
            qm = np.where(np.abs(im) > 1e-12, re / im, np.inf)
        return (np.log(np.maximum(qm, 1e-6)) - np.log(q)) * weights

    x0 = np.concatenate([np.log(tau0), np.log(delta0)])
    try:
        sol = least_squares(residual, x0, bounds=(x0 - 3.0, x0 + 3.0), max_nfev=400, xtol=1e-10, ftol=1e-10)
    except Exception:  # pragma: no cover - degenerate fit
        tau, dlt = _single_mechanism(q, f_ref)
        return _pack(q, f_ref, [tau], [dlt], (f_lo, f_hi), 0.0)
    tau = np.exp(sol.x[:n])
    dlt = np.exp(sol.x[n:])
    fitted = _pack(q, f_ref, tau, dlt, (f_lo, f_hi), 0.0)
    err = float(np.max(np.abs(np.log(np.maximum(fitted.quality(freqs), 1e-6)) - np.log(q))))
    return _pack(q, f_ref, tau, dlt, (f_lo, f_hi), err)


@dataclass
class RelaxationTables:
    """Per-Q tables for the device (one row per distinct Q value)."""

    q_values: np.ndarray          # (n_q,) distinct clipped Q
    qidx: np.ndarray              # (nzp, nxp) uint8 index into the tables
    tau: np.ndarray               # (n_q, L) float64
    delta: np.ndarray             # (n_q, L) float64, −αΔ under compensation
    modulus_ref: np.ndarray       # (n_q,) Re K_norm(f_ref)
    relax_a: np.ndarray           # (n_q, L) float32 exp(−dt/τ)
    fit_error: float = 0.0
    alpha_mechanisms: tuple[float, ...] = ()
    f_peak_mechanisms: tuple[float, ...] = ()
    extra: dict = field(default_factory=dict)


def distinct_q(qp: np.ndarray) -> np.ndarray:
    """The distinct clipped Q values a viscoacoustic model is fitted for."""
    return np.unique(np.clip(np.asarray(qp, dtype=np.float64).ravel(), 2.5, 1.0e5))


def prefit(qp: np.ndarray, f_ref: float, n_mechanisms: int, band_ratio: float) -> None:
    """Fit (and memoise) every distinct Q of a model ahead of propagator set-up."""
    for qv in distinct_q(qp)[:33]:
        if qv <= 1.0e4:
            fit_gsls(float(qv), f_ref, n_mechanisms=n_mechanisms, band_ratio=band_ratio)


def relaxation_tables(qp_padded: np.ndarray, dt: float, nt: int, *, f_ref: float, n_mechanisms: int,
                      band_ratio: float, compensation: bool, alpha_c: float, f_max: float | None,
                      gain_budget_db: float) -> RelaxationTables:
    """propagation.py:563-675 up to the per-cell expansion."""
    n = int(n_mechanisms)
    vals = np.clip(np.asarray(qp_padded, dtype=np.float64).ravel(), 2.5, 1.0e5)
    uniq = np.unique(vals)
    if uniq.size > 32:
        # The reference fits the median and then indexes past its one-row
        # table (propagation.py:627-628, 658), i.e. it cannot run such models.
        raise ERTMError(f"{uniq.size} distinct Q values; the viscoacoustic engine supports at most 32")
    tau = np.zeros((uniq.size, n))
    dlt = np.zeros((uniq.size, n))
    mref = np.zeros(uniq.size)
    fit_error = 0.0
    for i, qv in enumerate(uniq):
        if qv > 1.0e4:
            tau[i, :] = 1.0e-3
            dlt[i, :] = 0.0
            mref[i] = 1.0
            continue
        p = fit_gsls(float(qv), f_ref, n_mechanisms=n, band_ratio=band_ratio)
        fit_error = max(fit_error, p.fit_error)
        t = np.asarray(p.tau_sigma, dtype=np.float64)
        d = np.asarray(p.delta, dtype=np.float64)
        tau[i, : t.size] = t
        if t.size < n:
            tau[i, t.size:] = t[-1]
        dlt[i, : d.size] = d
        mref[i] = float(np.real(normalized_modulus(t, d, [f_ref])[0]))
    idx = np.searchsorted(uniq, vals).reshape(np.shape(qp_padded))
    if compensation:
        total = max(nt * dt, dt)
        gain = 10.0 ** (float(gain_budget_db) / 20.0)
        alpha_table = np.zeros((uniq.size, n))
        fpk_table = np.zeros((uniq.size, n))
        for i, qv in enumerate(uniq):
            fpk = np.sqrt(np.maximum(1.0 - dlt[i], 1e-6)) / (2.0 * np.pi * tau[i])
            fpk_table[i] = fpk
            keep = np.ones(n, dtype=bool) if f_max is None else fpk <= float(f_max)
            need = np.log(gain) * max(float(qv), 1.0) / (np.pi * np.maximum(fpk, 1e-6) * total)
            alpha = np.where(keep, np.minimum(float(alpha_c), need), 0.0)
            alpha_table[i] = alpha
            dlt[i] = -alpha * dlt[i]
        alphas = tuple(float(v) for v in np.mean(alpha_table, axis=0))
        fpeaks = tuple(float(v) for v in np.mean(fpk_table, axis=0))
    else:
        alphas = tuple(float(alpha_c) for _ in range(n))
        fpeaks = tuple(float(v) for v in np.mean(np.sqrt(np.maximum(1.0 - dlt, 1e-6)) / (2.0 * np.pi * tau), axis=0))
    relax_a = np.exp(-dt / tau).astype(np.float32)
    return RelaxationTables(q_values=uniq, qidx=idx.astype(np.uint8), tau=tau, delta=dlt, modulus_ref=mref,
                            relax_a=relax_a, fit_error=fit_error, alpha_mechanisms=alphas,
                            f_peak_mechanisms=fpeaks)
