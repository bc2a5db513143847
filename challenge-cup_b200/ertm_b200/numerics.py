"""Host-side numerics for setting up the device path.

Only set-up arithmetic lives here (stencil coefficients, CFL limit, CPML
profiles, source wavelets, the record sinc resampler used before a shot is
uploaded).  Every per-cell, per-step operation runs in the CUDA library.
Formulas follow ertm/numerics.py; they are evaluated with NumPy in the same
order so the float32 profiles equal the reference's bit for bit.
"""

from __future__ import annotations

import numpy as np

#: Staggered first-derivative coefficients (Levander 1988; numerics.py:35-40).
STAGGERED_COEFFICIENTS: dict[int, tuple[float, ...]] = {
    2: (1.0,),
    4: (9.0 / 8.0, -1.0 / 24.0),
    6: (75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0),
    8: (1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0),
}
SUPPORTED_ORDERS = tuple(sorted(STAGGERED_COEFFICIENTS))


def staggered_coefficients(order: int) -> tuple[float, ...]:
    try:
        return STAGGERED_COEFFICIENTS[int(order)]
    except (KeyError, TypeError) as exc:
        raise ValueError(f"unsupported order {order!r}; choose from {SUPPORTED_ORDERS}") from exc


def coefficient_l1(order: int) -> float:
    return float(sum(abs(c) for c in staggered_coefficients(order)))


def ghost_width(order: int) -> int:
    """Padding on each side of the grid: half stencil + 1 (numerics.py:60-62)."""
    return len(staggered_coefficients(order)) + 1


def cfl_dt(vmax: float, dx: float, dz: float, order: int, safety: float = 0.5) -> float:
    """Δt ≤ safety / (vmax·√((C/dx)² + (C/dz)²)) (numerics.py:314-326)."""
    if vmax <= 0:
        raise ValueError(f"vmax must be positive, got {vmax}")
    c = coefficient_l1(order)
    return float(safety / (vmax * np.hypot(c / dx, c / dz)))


def points_per_wavelength(vmin: float, f0: float, spacing: float) -> float:
    return float(vmin / (f0 * spacing)) if vmin > 0 and f0 > 0 else 0.0


def cpml_profile(length: int, spacing: float, npml: int, dt: float, vmax: float, *, alpha_max: float,
                 sides: tuple[bool, bool] = (True, True), enabled: bool = True
                 ) -> tuple[np.ndarray, np.ndarray, int]:
    """CFS-PML recursion coefficients of one padded axis (numerics.py:155-219).

    Quadratic σ profile with R = 1e-5, κ ≡ 1, α falling linearly from
    α_max at the outer edge to 0 at the inner edge; strips counted from the
    padded edge, width clamped to length//3.  Returns float32 ``(b, a)`` and
    the strip width.
    """
    if length < 2:
        raise ValueError("PML axis needs at least 2 cells")
    n = int(max(1, min(npml, length // 3)))
    sigma = np.zeros(length, dtype=np.float64)
    alpha = np.zeros(length, dtype=np.float64)
    depth = max(n * spacing, spacing)
    sigma_max = -(2 + 1) * vmax * np.log(max(1e-5, 1e-12)) / (2.0 * depth)
    d = (n - np.arange(n, dtype=np.float64)) / n
    shape = d**2
    if enabled and sides[0]:
        sigma[:n] = sigma_max * shape
        alpha[:n] = float(alpha_max) * (1.0 - d)
    if enabled and sides[1]:
        sigma[length - n:] = sigma_max * shape[::-1]
        alpha[length - n:] = float(alpha_max) * (1.0 - d[::-1])
    denom = sigma * 1.0 + 1.0 * 1.0 * alpha          # σκ + κ²α with κ = 1
    b = np.exp(-(sigma / 1.0 + alpha) * dt)
    a = np.zeros_like(sigma)
    ok = denom > 0
    a[ok] = sigma[ok] / denom[ok] * (b[ok] - 1.0)
    return b.astype(np.float32), a.astype(np.float32), n


def ricker(t: np.ndarray, f0: float, t0: float = 0.0) -> np.ndarray:
    """Ricker wavelet, peak 1 at t0 (numerics.py:466-469)."""
    arg = np.pi * float(f0) * (np.asarray(t) - float(t0))
    return ((1.0 - 2.0 * arg**2) * np.exp(-arg**2)).astype(np.float32)


def gaussian_pulse(t: np.ndarray, f0: float, t0: float = 0.0) -> np.ndarray:
    """numerics.py:472-475."""
    arg = np.pi * float(f0) * (np.asarray(t) - float(t0))
    return np.exp(-0.5 * arg**2).astype(np.float32)


def resample_sinc(data: np.ndarray, dt_in: float, dt_out: float, *, axis: int = 0, half_length: int = 8,
                  beta: float = 8.6) -> np.ndarray:
    """Kaiser-windowed sinc resampling of a record to the propagation dt.

    Host pre-pass of the record preparation (numerics.py:337-392), run once
    per shot before the record is uploaded.
    """
    a = np.asarray(data, dtype=np.float64)
    if dt_in <= 0 or dt_out <= 0:
        raise ValueError("dt_in / dt_out must be positive")
    squeeze = a.ndim == 1
    if squeeze:
        a = a[:, None]
    elif a.ndim != 2:
        raise ValueError(f"only 1-D/2-D data, got {a.ndim}-D")
    if axis == 1:
        a = a.T
    n_in = a.shape[0]
    if n_in < 3:
        raise ValueError(f"too few samples ({n_in}) to interpolate")
    n_out = int(np.floor((n_in - 1) * dt_in / dt_out + 1e-9)) + 1
    pos = np.arange(n_out, dtype=np.float64) * (dt_out / dt_in)
    taps = np.arange(-half_length + 1, half_length + 1)
    off = np.floor(pos).astype(np.int64)[:, None] + taps[None, :]
    w = np.sinc(pos[:, None] - off) * np.kaiser(2 * half_length, beta)[None, :]
    s = w.sum(axis=1, keepdims=True)
    s[s == 0] = 1.0
    w /= s
    out = np.ascontiguousarray(np.einsum("ot,ots->os", w, a[np.clip(off, 0, n_in - 1)]))
    if squeeze:
        out = out[:, 0]
    return out.T if axis == 1 else out


def lowpass_wavenumber(field: np.ndarray, dx: float, dz: float, cutoff_fraction: float = 0.85) -> np.ndarray:
    """Wavenumber low-pass (numerics.py:424-442) on the device.

    ``Re(ifft2(fft2(field) · taper))`` with the radial taper
    ``clip(1 − (k − cutoff)/0.15, 0, 1)`` over Nyquist-normalised wavenumbers.
    The CUDA transforms follow numpy.fft's arithmetic, so the float64 result
    equals the reference's bit for bit.  Returns a new float64 array."""
    if not 0.0 < cutoff_fraction <= 1.0:
        raise ValueError(f"cutoff_fraction must lie in (0, 1], got {cutoff_fraction}")
    from . import _lib
    a = np.ascontiguousarray(field, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError(f"lowpass_wavenumber takes a 2-D field, got {a.ndim}-D")
    out = np.empty_like(a)
    nz, nx = a.shape
    _lib.check(_lib.lib().ertm_lowpass_wavenumber(nz, nx, float(dx), float(dz), float(cutoff_fraction),
                                                  a.ctypes.data, out.ctypes.data, None), "lowpass_wavenumber")
    return out
