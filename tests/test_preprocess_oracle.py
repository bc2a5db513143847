"""Record preprocessing: the oracle restatement against the reference's own
outputs (tests/golden/preprocess.npz, made by tests/golden/make_golden.py)."""

from __future__ import annotations

import numpy as np

import oracle as orc
from helpers import load


def test_oracle_rotation_resampling_mute_taper_match_golden():
    fx = load("preprocess")
    comps = {n: fx[f"in_{n}"] for n in ("p", "vx", "vz")}
    rot = orc.rotate_components(comps, 30.0)
    for n in comps:
        assert np.array_equal(rot[n], fx[f"rot_{n}"]), n
    dt = float(fx["dt"])
    for tag, dt_out in (("up", 3e-4), ("down", 5.5e-4)):
        for n in comps:
            got = orc.resample_sinc(comps[n].astype(np.float64), dt, dt_out).astype(np.float32)
            assert np.allclose(got, fx[f"res_{tag}_{n}"], rtol=0, atol=1e-6 * np.abs(fx[f"res_{tag}_{n}"]).max())
    t = np.arange(int(fx["nt"])) * dt
    x, z, f0, delay, _ = fx["src"]
    w = orc.mute_weights(t, fx["rx"], x, f0, delay, 2100.0)
    for n in comps:
        assert np.array_equal((comps[n].astype(np.float64) * w).astype(np.float32), fx[f"mute_{n}"]), n
        assert np.array_equal(orc.taper_ends(comps[n], 0.05).astype(np.float32), fx[f"taper_{n}"]), n


def test_oracle_q_filter_matches_golden():
    fx = load("qcomp")
    dt = float(fx["dt"])
    got = orc.stft_filter(fx["data"], dt, lambda tc, f: orc.q_attenuation_response(f, max(tc, 1e-6), 50.0, 30.0),
                          nperseg=64)
    np.testing.assert_allclose(got, fx["attenuated"], rtol=0, atol=1e-12 * np.abs(fx["attenuated"]).max())
    got = orc.stft_filter(fx["data"][:, 0], dt, lambda tc, f: orc.q_attenuation_response(f, max(tc, 1e-6), 80.0,
                                                                                             30.0), nperseg=96)
    np.testing.assert_allclose(got, fx["trace"], rtol=0, atol=1e-12 * np.abs(fx["trace"]).max())
