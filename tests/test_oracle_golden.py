"""Pin the CPU oracle against golden vectors made by the reference itself.

Fixtures were generated by ``tests/golden/make_golden.py`` from the
reference's own ``ertm`` code.  The oracle agrees with them bit for bit:
propagation of all three engines (the compensated viscoacoustic run with its
FFT low-pass included), migrated images and stacks.  Only set-up values that
go through NumPy's vectorised transcendental functions on the host (CPML
``exp`` profiles, the sinc/Kaiser resampling weights, the GSLS least-squares
fit) carry a tolerance, stated per assertion: those functions may round
differently in the last place on another CPU.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from helpers import (MIGRATE_CASES, PROPAGATION_CASES, imaging_from, load, model_from,
                     q_from, q_options_for_migrate, receivers_from, rel_l2, solver_from,
                     source_from)


def test_derivatives_bit_exact():
    fx = load("numerics")
    f = fx["deriv_in"]
    for order in (2, 4, 6, 8):
        for axis in (0, 1):
            h = 7.5 if axis == 1 else 5.0
            assert np.array_equal(orc.stagger_diff(f, axis, True, h, order), fx[f"dplus_o{order}_a{axis}"])
            assert np.array_equal(orc.stagger_diff(f, axis, False, h, order), fx[f"dminus_o{order}_a{axis}"])


def test_cpml_profiles_and_scalars():
    fx = load("numerics")
    cases = [(61, 10.0, 20, 1e-3, 3000.0, (True, True), True),
             (41, 5.0, 40, 3e-4, 4500.0, (False, True), True),
             (30, 10.0, 8, 5e-4, 2500.0, (True, True), False)]
    for i, (n, h, npml, dt, vmax, sides, en) in enumerate(cases):
        ax = orc.PMLAxis(n, h, npml, dt, vmax, alpha_max=2.0 * np.pi * 25.0, sides=sides, enabled=en)
        assert ax.npml == int(fx[f"cpml{i}_npml"])
        # exp() on float64 then cast to float32: identical unless NumPy's exp differs by an ulp.
        np.testing.assert_allclose(ax.b, fx[f"cpml{i}_b"], rtol=2e-7, atol=0)
        np.testing.assert_allclose(ax.a, fx[f"cpml{i}_a"], rtol=2e-7, atol=1e-12)
    cfl = [orc.cfl_dt(3000.0, 10.0, 10.0, 8, 0.5), orc.cfl_dt(4500.0, 5.0, 5.0, 8, 0.55),
           orc.cfl_dt(4000.0, 5.0, 5.0, 4, 0.5)]
    assert np.array_equal(np.array(cfl), fx["cfl"])
    np.testing.assert_allclose(orc.ricker(np.arange(300) * 1e-3, 15.0, 0.08), fx["ricker"], rtol=0, atol=1e-7)
    assert np.array_equal(orc.laplacian(fx["img_in"], 10.0, 5.0), fx["laplacian"])
    assert np.array_equal(orc.lowpass_wavenumber(fx["img_in"], 10.0, 5.0, 0.85), fx["lowpass"])
    assert np.array_equal(orc.bilinear(fx["deriv_in"], fx["bil_z"], fx["bil_x"]), fx["bilinear"])
    np.testing.assert_allclose(orc.resample_sinc(fx["resample_in"], 4e-4, 2.5e-4), fx["resample"],
                               rtol=0, atol=1e-12)


def test_gsls_fit_matches_reference():
    fx = load("gsls")
    for n in (1, 3):
        for i, q in enumerate(fx["q"]):
            fit = orc.fit_gsls(float(q), 30.0, n_mechanisms=n, band_ratio=1.5)
            k = len(fit.tau_sigma)
            # least-squares iterates in float64; the fit is reproduced to ~1e-12.
            np.testing.assert_allclose(fit.tau_sigma, fx[f"tau_n{n}"][i, :k], rtol=1e-9)
            np.testing.assert_allclose(fit.delta, fx[f"delta_n{n}"][i, :k], rtol=1e-9)
            mref = float(np.real(orc.normalized_modulus(fit.tau_sigma, fit.delta, [30.0])[0]))
            np.testing.assert_allclose(mref, fx[f"mref_n{n}"][i], rtol=1e-12)


def _run_oracle_propagation(fx: dict):
    meta = fx["meta"]
    dt, nt, order, npml = fx["spec"]
    spec = orc.Spec(dt=float(dt), nt=int(nt), order=int(order), npml=int(npml), dtype=meta["dtype"],
                    boundary=meta["boundary"])
    prop = orc.build_oracle(model_from(fx), spec, meta["engine"], q_from(meta["q"]))
    prop.set_source(source_from(fx, meta["mechanism"]))
    prop.set_receivers(receivers_from(fx))
    names = meta["names"]
    rec = {n: np.zeros((int(nt), len(fx["rx"])), np.float32) for n in names}
    for t in range(int(nt)):
        if meta["inject_every"] and t % meta["inject_every"] == 0:
            for n in names:
                prop.inject(n, fx["inj_values"][t])
        prop.step(float(fx["wavelet"][t]))
        s = prop.sample(names)
        for n in names:
            rec[n][t] = s[n]
    return prop, rec


@pytest.mark.parametrize("case", PROPAGATION_CASES)
def test_oracle_propagation_matches_reference(case):
    fx = load(case)
    prop, rec = _run_oracle_propagation(fx)
    st = prop.state()
    meta = fx["meta"]
    for k, v in st.items():
        key = f"state_{k.replace(':', '_')}"
        assert key in fx, key
        assert np.array_equal(v, fx[key]), (case, k, rel_l2(v, fx[key]))
    for n, r in rec.items():
        assert np.array_equal(r, fx[f"rec_{n}"]), (case, n)
    assert prop.state_bytes() == meta["state_bytes"]
    if meta["engine"] == "elastic":
        for sep in ("stress", "divcurl"):
            for k, v in prop.image_fields(sep).items():
                assert np.array_equal(v, fx[f"img_{sep}_{k}"])
    if meta["engine"] == "viscoacoustic":
        assert np.array_equal(prop.k_relaxed, fx["k_relaxed"])
        assert np.array_equal(prop.b, fx["relax_b"])
        assert prop.clipped == int(fx["clipped"])
        assert prop.lowpass_steps == int(fx["lowpass_steps"])


@pytest.mark.parametrize("case", MIGRATE_CASES)
def test_oracle_migrate_matches_reference(case):
    fx = load(case)
    meta = fx["meta"]
    comps = {k[len("shot_"):]: v for k, v in fx.items() if k.startswith("shot_") and k != "shot_dt"}
    img, terms = orc.migrate(comps, float(fx["shot_dt"]), source_from(fx), receivers_from(fx),
                             model_from(fx), solver_from(meta), imaging_from(meta),
                             q_options_for_migrate(meta["q"]), return_terms=True)
    assert terms["interval"] == meta["checkpoints"]["interval"]
    assert terms["n_states"] == meta["checkpoints"]["n_states"]
    assert terms["start_step"] == meta["start_step"]
    assert np.array_equal(img, fx["image"]), rel_l2(img, fx["image"])


def test_stack_images():
    fx = load("stack")
    assert np.array_equal(orc.stack_images(list(fx["images"])), fx["stacked"])
