"""Record preprocessing on the device against the reference's own outputs
(tests/golden/preprocess.npz)."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import load, model_from

pytestmark = pytest.mark.gpu


def _shot(fx):
    from ertm_b200.types import ReceiverSpec, ShotRecord, SourceSpec
    x, z, f0, delay, amp = fx["src"]
    comps = {n: fx[f"in_{n}"] for n in ("p", "vx", "vz")}
    dt = float(fx["dt"])
    return ShotRecord(data=comps["p"], dt=dt, t=np.arange(int(fx["nt"])) * dt,
                      receivers=ReceiverSpec(x=fx["rx"], z=fx["rz"]),
                      source=SourceSpec(x=float(x), z=float(z), f0=float(f0), delay=float(delay)), components=comps)


def _close(a, b, rel=1e-6):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and a.dtype == np.float32
    assert np.max(np.abs(a.astype(np.float64) - b)) <= rel * np.max(np.abs(b)), np.max(np.abs(a - b))


def test_rotation_and_taper_bit_exact():
    from ertm_b200 import preprocess as pre
    fx = load("preprocess")
    shot = _shot(fx)
    rot = pre.rotate_components(shot.components, 30.0)
    for n in ("p", "vx", "vz"):
        assert np.array_equal(rot[n], fx[f"rot_{n}"]), n
    tp = pre.taper_record_ends(shot, 0.05)
    for n in ("p", "vx", "vz"):
        assert np.array_equal(tp.components[n], fx[f"taper_{n}"]), n
    assert np.array_equal(tp.data, fx["taper_data"].astype(np.float32))


def test_resampling_and_mute_match_reference():
    from ertm_b200 import preprocess as pre
    fx = load("preprocess")
    shot = _shot(fx)
    for tag, dt_out in (("up", 3e-4), ("down", 5.5e-4)):
        r = pre.resample_shot(shot, dt_out)
        for n in ("p", "vx", "vz"):
            _close(r.components[n], fx[f"res_{tag}_{n}"])
        assert r.dt == dt_out and r.t.size == fx[f"res_{tag}_p"].shape[0]
    m = pre.mute_direct_wave(shot, 2100.0)
    for n in ("p", "vx", "vz"):
        _close(m.components[n], fx[f"mute_{n}"])


def test_prepare_shot_matches_reference():
    from ertm_b200 import preprocess as pre
    fx = load("preprocess")
    ps = pre.prepare_shot(_shot(fx), model=model_from(fx), record_dt=3.5e-4, rotation_deg=25.0, mute=True,
                          taper_fraction=0.05)
    assert ps.dt == float(fx["prep_dt"])
    for n in ("p", "vx", "vz"):
        _close(ps.components[n], fx[f"prep_{n}"])


def test_migrate_resamples_records_on_the_device():
    """A record at another sampling interval goes through the device sinc
    resampling in RTMImager; the image matches migrating the record the
    oracle resampled."""
    from ertm_b200 import preprocess as pre
    from ertm_b200.numerics import resample_sinc as host_resample
    fx = load("preprocess")
    a = fx["in_p"].astype(np.float64)
    dev = pre.resample_sinc(a, 4e-4, 3.3e-4)
    host = host_resample(a, 4e-4, 3.3e-4).astype(np.float32)
    _close(dev, host)
