"""Form (a): the device images (float32 wavefields; float64 or
Kahan-compensated float32 imaging sums) against images of the oracle run in
float64 wavefields, on seeded shots of each benchmark configuration.

The float64 images are committed under tests/precision/ (made on the CPU by
tests/precision/make_fp64.py, every ``step``-th pixel), and so are the
oracle's float32 images (the reference's own precision, ``<config>_f32``).
The device computes the same shots from the same seeded inputs here.

What is checked:

* parity: with float64 imaging sums the device images EQUAL the reference's
  float32 images bit for bit, at full size, for every configuration that has
  them (the compensated viscoacoustic one included); Kahan float32 sums stay
  within 1e-6 of them;
* precision: the device's error against float64 is therefore exactly the
  reference's own float32 error.  It is ≤ 1e-4 for the acoustic and uneven
  configurations (asserted).  For the elastic (PS 2.4e-4) and compensated
  viscoacoustic (3.1e-4, shot 10) configurations float32 wave propagation
  itself, in the reference as on the device, exceeds 1e-4; there the test
  asserts the equality with the reference's error and reports the number.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

from helpers import rel_l2

PREC = Path(__file__).resolve().parent / "precision"
sys.path.insert(0, str(PREC))
from make_fp64 import CASES, case_workloads  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 1e-4
KAHAN_TO_F32 = 1e-6
CONFIGS = [c for c in CASES if (PREC / f"{c}.npz").exists()]


@pytest.mark.parametrize("accumulation", ["fp64", "kahan"])
@pytest.mark.parametrize("config", CONFIGS)
def test_image_error_against_fp64_oracle(config, accumulation):
    from ertm_b200 import RTMImager, workloads
    from ertm_b200.stacking import stack_images
    with np.load(PREC / f"{config}.npz") as z:
        fx = {k: z[k] for k in z.files}
    meta = json.loads(str(fx["meta"]))
    step = int(meta["step"])
    per_mode: dict[str, list] = {}
    for k, wl in enumerate(case_workloads(config)):
        base, solver = workloads.imager_for(wl)
        imager = RTMImager(base.config, solver, base.q_config, accumulation=accumulation)
        record = workloads.synthesize(wl, solver, wl.sources)[0]
        for res in imager.migrate_modes(record, wl.model, modes=wl.modes):
            per_mode.setdefault(res.mode, []).append((k, res))
    # where the oracle's float32 images exist too (<config>_f32.npz, the
    # reference's own precision), report the device against them and the
    # reference's own float32 error against float64
    f32 = None
    if (PREC / f"{config}_f32.npz").exists():
        with np.load(PREC / f"{config}_f32.npz") as z:
            f32 = {k: z[k] for k in z.files}
    errors, vs_f32, ref_err = {}, {}, {}
    for m, results in per_mode.items():
        if meta["stacked"]:
            keyed = [(m, stack_images([r for _, r in results]).image[::step, ::step])]
        else:
            keyed = [(f"{m}_{k}", r.image[::step, ::step]) for k, r in results]
        for key, img in keyed:
            errors[key] = rel_l2(img, fx[key])
            if f32 is not None:
                vs_f32[key] = rel_l2(img, f32[key])
                ref_err[key] = rel_l2(f32[key], fx[key])
    print(f"\nprecision {config} {accumulation}: " + json.dumps(errors)
          + ("" if f32 is None else " device vs float32 oracle: " + json.dumps(vs_f32)
             + " float32 oracle vs float64: " + json.dumps(ref_err)))
    if f32 is not None:
        if accumulation == "fp64":
            assert all(v == 0.0 for v in vs_f32.values()), vs_f32
            assert errors == ref_err, (errors, ref_err)
        else:
            assert max(vs_f32.values()) <= KAHAN_TO_F32, vs_f32
    float32_exceeds = f32 is not None and max(ref_err.values()) > TOL
    if not float32_exceeds:
        assert max(errors.values()) <= TOL, errors
