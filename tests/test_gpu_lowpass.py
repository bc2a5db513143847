"""The device wavenumber low-pass against NumPy's, bit for bit.

``lowpass_wavenumber`` (numerics.py:424-442) runs fft2 → radial taper →
ifft2 → real part.  The CUDA line transforms reproduce numpy.fft's
arithmetic (pocketfft's plans and operation order), so the float64 results
must be identical.  The shapes cover every pass the plans use: radix
2/3/4/5/7/8/11 passes, the generic pass of a larger prime factor, Bluestein
lengths (primes such as 811 and 2011, the padded widths of the 2001×801
viscoacoustic grid), and a Bluestein length whose work buffers do not fit
in shared memory (4106 → inner length 8232, the padded width of a
4096-column grid).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 3), (7, 11), (16, 24), (40, 50), (53, 71), (13, 169), (101, 97), (64, 121),
          (211, 311), (120, 360), (811, 2011), (2058, 4106)]


@pytest.mark.parametrize("nz,nx", SHAPES)
def test_lowpass_wavenumber_bit_exact(nz, nx):
    from ertm_b200 import _lib
    from ertm_b200.numerics import lowpass_wavenumber
    _lib.lib()
    rng = np.random.default_rng(nz * 10007 + nx)
    field = rng.standard_normal((nz, nx))
    field[:, : nx // 3] = 0.0                      # silent region, as ahead of a wavefront
    for cutoff, dz, dx in ((0.85, 10.0, 5.0), (0.35, 5.0, 5.0)):
        got = lowpass_wavenumber(field, dx, dz, cutoff)
        want = orc.lowpass_wavenumber(field, dx, dz, cutoff)
        assert np.array_equal(got, want), (nz, nx, cutoff, float(np.max(np.abs(got - want))))


# threads per CTA of the line transforms (0: the per-length choice); every
# count must give the same bits
LINE_THREADS = [64, 96, 128, 192, 288, 512, 640, 1024]


@pytest.mark.parametrize("threads", LINE_THREADS)
def test_lowpass_bit_exact_for_every_thread_count(threads):
    from ertm_b200 import _lib
    from ertm_b200.numerics import lowpass_wavenumber
    L = _lib.lib()
    _lib.check(L.ertm_set_line_threads(threads), "line threads")
    try:
        for nz, nx in ((13, 169), (53, 71), (101, 97), (211, 311), (811, 2011), (2058, 4106)):
            rng = np.random.default_rng(nz + 7 * nx)
            field = rng.standard_normal((nz, nx))
            got = lowpass_wavenumber(field, 5.0, 10.0, 0.55)
            want = orc.lowpass_wavenumber(field, 5.0, 10.0, 0.55)
            assert np.array_equal(got, want), (threads, nz, nx)
    finally:
        _lib.check(L.ertm_set_line_threads(0), "line threads")


def test_line_threads_knob_rejects_bad_values():
    from ertm_b200 import _lib
    L = _lib.lib()
    assert L.ertm_set_line_threads(100) != 0
    assert L.ertm_set_line_threads(1056) != 0
    assert L.ertm_set_line_threads(32) != 0
    assert L.ertm_set_line_threads(0) == 0


def test_lowpass_wavenumber_of_float32_field_device_resident():
    """A float32 field in place on the device (the compensated visco path's
    input form goes through the same transforms)."""
    import torch

    from ertm_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(3)
    f32 = rng.standard_normal((57, 63)).astype(np.float32)
    d = torch.from_numpy(f32.astype(np.float64)).cuda()
    _lib.check(L.ertm_lowpass_wavenumber(57, 63, 7.5, 5.0, 0.6, d.data_ptr(), d.data_ptr(), None), "lowpass")
    want = orc.lowpass_wavenumber(f32, 7.5, 5.0, 0.6)
    assert np.array_equal(d.cpu().numpy(), want)


def test_lowpass_rejects_bad_cutoff():
    from ertm_b200.numerics import lowpass_wavenumber
    with pytest.raises(ValueError):
        lowpass_wavenumber(np.zeros((4, 4)), 1.0, 1.0, 0.0)
