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
