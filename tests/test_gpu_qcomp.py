"""Data-domain Q filter on the device against the reference's own outputs
(tests/golden/qcomp.npz): cuFFT double vs pocketfft, bound 1e-10 relative."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import load

pytestmark = pytest.mark.gpu


def _close(a, b, rel=1e-10):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    assert np.max(np.abs(a - b)) <= rel * np.max(np.abs(b)), np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_compensator_and_attenuation_match_reference():
    from ertm_b200.config import QConfig
    from ertm_b200.qcomp import QCompensator, attenuate_record
    fx = load("qcomp")
    dt = float(fx["dt"])
    comp = QCompensator(config=QConfig(enabled=True, model="filter", alpha_c=0.8, gain_cap=30.0, f_ref=30.0),
                        q_value=60.0)
    _close(comp(fx["data"].astype(np.float64), dt), fx["compensated"])
    _close(attenuate_record(fx["data"], dt, 50.0, f_ref=30.0, nperseg=64), fx["attenuated"])
    _close(attenuate_record(fx["data"][:, 0], dt, 80.0, nperseg=96), fx["trace"])


@pytest.mark.parametrize("n,ntr,nperseg", [(3, 2, 128), (5, 1, 128), (9, 3, 8), (130, 4, 64), (257, 2, 128),
                                           (1000, 5, 96)])
def test_time_varying_filter_edges_match_oracle(n, ntr, nperseg):
    """Records shorter than a frame (no frame at all below 4 samples), ragged
    last frames and odd frame lengths, against the oracle's overlap-add."""
    from oracle import ertm_oracle as orc
    from ertm_b200.qcomp import q_response, time_varying_filter
    x = np.random.default_rng(n).normal(size=(n, ntr))
    fn = lambda tc, f: q_response(f, max(tc, 1e-6), 40.0, 25.0)  # noqa: E731
    got = time_varying_filter(x, 2e-3, fn, nperseg=nperseg)
    want = orc.stft_filter(x, 2e-3, lambda tc, f: orc.q_attenuation_response(f, max(tc, 1e-6), 40.0, 25.0),
                           nperseg=nperseg)
    assert got.shape == want.shape
    if n < 4:
        assert not np.any(got) and not np.any(want)
    else:
        _close(got, want, rel=1e-12)


def test_q_filter_rejects_bad_input():
    from ertm_b200.qcomp import DataError, attenuate_record, time_varying_filter
    with pytest.raises(DataError):
        attenuate_record(np.zeros((10, 2, 2)), 1e-3, 50.0)
    with pytest.raises(DataError):
        attenuate_record(np.zeros((10, 2)), 1e-3, -5.0)
    with pytest.raises(DataError):
        time_varying_filter(np.zeros((64, 2)), 1e-3, lambda tc, f: np.ones(3), nperseg=16)
