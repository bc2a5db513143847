"""CPU-only checks of the host side: library exports, set-up arithmetic,
schedules and error behaviour (no kernel is launched here)."""

from __future__ import annotations

import ctypes
import dataclasses
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from helpers import load

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    from ertm_b200 import _lib
    header = (ROOT / "include" / "ertm_b200.h").read_text()
    declared = set(re.findall(r"\b(ertm_[a-z0-9_]+)\s*\(", header))
    so = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [name for name in sorted(declared) if not hasattr(so, name)]
    assert not missing, missing
    assert declared >= set(_lib.exported_symbols())
    assert so.ertm_version() >= 1


def test_cpml_profiles_equal_oracle_and_golden():
    from ertm_b200.numerics import cpml_profile
    fx = load("numerics")
    cases = [(61, 10.0, 20, 1e-3, 3000.0, (True, True), True), (41, 5.0, 40, 3e-4, 4500.0, (False, True), True),
             (30, 10.0, 8, 5e-4, 2500.0, (True, True), False)]
    for i, (n, h, npml, dt, vmax, sides, en) in enumerate(cases):
        b, a, width = cpml_profile(n, h, npml, dt, vmax, alpha_max=2 * np.pi * 25.0, sides=sides, enabled=en)
        ax = orc.PMLAxis(n, h, npml, dt, vmax, alpha_max=2 * np.pi * 25.0, sides=sides, enabled=en)
        assert np.array_equal(b, ax.b) and np.array_equal(a, ax.a)
        assert width == int(fx[f"cpml{i}_npml"])
        np.testing.assert_allclose(b, fx[f"cpml{i}_b"], rtol=2e-7)


def test_wavelet_and_cfl_match_reference():
    from ertm_b200 import numerics as num
    fx = load("numerics")
    np.testing.assert_allclose(num.ricker(np.arange(300) * 1e-3, 15.0, 0.08), fx["ricker"], atol=1e-7, rtol=0)
    assert num.cfl_dt(3000.0, 10.0, 10.0, 8, 0.5) == fx["cfl"][0]
    assert num.cfl_dt(4500.0, 5.0, 5.0, 8, 0.55) == fx["cfl"][1]
    np.testing.assert_allclose(num.resample_sinc(fx["resample_in"], 4e-4, 2.5e-4), fx["resample"], atol=1e-12)


def test_gsls_fit_matches_reference_golden():
    from ertm_b200.viscoelastic import fit_gsls, normalized_modulus
    fx = load("gsls")
    for n in (1, 3):
        for i, q in enumerate(fx["q"]):
            p = fit_gsls(float(q), 30.0, n_mechanisms=n, band_ratio=1.5)
            k = len(p.tau_sigma)
            np.testing.assert_allclose(p.tau_sigma, fx[f"tau_n{n}"][i, :k], rtol=1e-9)
            np.testing.assert_allclose(p.delta, fx[f"delta_n{n}"][i, :k], rtol=1e-9)
            m = float(np.real(normalized_modulus(p.tau_sigma, p.delta, [30.0])[0]))
            np.testing.assert_allclose(m, fx[f"mref_n{n}"][i], rtol=1e-12)


def test_relaxation_tables_reproduce_reference_coefficients():
    """Host tables + the device's per-cell formula, evaluated here in NumPy,
    give the reference's a_l and b_l (propagation.py:660-667)."""
    from ertm_b200.viscoelastic import relaxation_tables
    fx = load("visco_comp_free")
    meta = fx["meta"]
    q = meta["q"]
    pad = 5
    qp = np.pad(fx["m_qp"].astype(np.float32), pad, mode="edge")
    t = relaxation_tables(qp, float(fx["spec"][0]), int(fx["spec"][1]), f_ref=q["f_ref"],
                          n_mechanisms=q["n_mechanisms"], band_ratio=q["band_ratio"],
                          compensation=q["compensation"], alpha_c=q["alpha_c"], f_max=q["f_max"],
                          gain_budget_db=q["gain_budget_db"])
    rho = np.pad(fx["m_rho"], pad, mode="edge")
    vp = np.pad(fx["m_vp"], pad, mode="edge")
    kappa = rho * vp * vp
    kr = (kappa / t.modulus_ref[t.qidx]).astype(np.float32)
    np.testing.assert_allclose(kr, fx["k_relaxed"], rtol=1e-7)
    a = np.moveaxis(t.relax_a[t.qidx], -1, 0)
    np.testing.assert_allclose(a, fx["relax_a"], rtol=1e-7)
    b = (kr[None] * np.moveaxis(t.delta[t.qidx], -1, 0) * (1.0 - a) * np.moveaxis(t.tau[t.qidx], -1, 0)
         / float(fx["spec"][0])).astype(np.float32)
    np.testing.assert_allclose(b, fx["relax_b"], rtol=1e-6, atol=1e-3)


def test_relaxation_rejects_more_than_32_q_values():
    from ertm_b200.exceptions import ERTMError
    from ertm_b200.viscoelastic import relaxation_tables
    qp = np.linspace(20.0, 200.0, 40, dtype=np.float32)[None, :].repeat(3, 0)
    with pytest.raises(ERTMError):
        relaxation_tables(qp, 1e-3, 10, f_ref=30.0, n_mechanisms=3, band_ratio=1.5, compensation=False,
                          alpha_c=1.0, f_max=None, gain_budget_db=40.0)


def test_checkpoint_interval_formula_matches_golden_runs():
    from ertm_b200.imaging import checkpoint_interval
    for case in ("mig_acoustic_zerolag", "mig_elastic_pp_divcurl", "mig_visco_comp"):
        meta = load(case)["meta"]
        nx, nz = 51, 41
        pad = 5
        n_fields = {"acoustic": 3, "elastic": 5, "viscoacoustic": 7}[meta["engine"]]
        per = n_fields * (nz + 2 * pad) * (nx + 2 * pad) * 4
        assert checkpoint_interval(meta["nt"], per, meta["checkpoint_mb"]) == meta["checkpoints"]["interval"]


def test_spec_stability_and_config_errors():
    from ertm_b200 import ConfigError, ImagingConfig, SolverConfig, SolverError
    from ertm_b200.propagation import PropagationSpec, check_stability
    from ertm_b200.types import ElasticModel, GridSpec
    g = GridSpec(nx=121, nz=91, dx=10.0, dz=10.0)
    sh = g.shape
    m = ElasticModel(grid=g, vp=np.full(sh, 4000.0, np.float32), vs=np.full(sh, 1700.0, np.float32),
                     rho=np.full(sh, 2400.0, np.float32), qp=np.full(sh, 100.0, np.float32),
                     qs=np.full(sh, 50.0, np.float32))
    with pytest.raises(SolverError):
        check_stability(m, PropagationSpec(dt=2e-3, nt=10, order=8, npml=8))
    check_stability(m, PropagationSpec(dt=4e-4, nt=10, order=8, npml=8))
    assert PropagationSpec.from_config(SolverConfig(), m).npml == 11   # min(20, max(8, 91//8))
    with pytest.raises(ConfigError):
        ImagingConfig(condition="bogus").validate()
    with pytest.raises(ConfigError):
        SolverConfig(npml=2).validate()
    with pytest.raises(ValueError):
        PropagationSpec(dt=1e-3, nt=10, boundary="wall")


def test_product_fails_loudly_without_a_device():
    """No CPU fallback: without a B200 the first propagator raises SolverError."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ertm_b200 import SolverError
    from ertm_b200.propagation import PropagationSpec, build_propagator
    from ertm_b200.types import ElasticModel, GridSpec
    g = GridSpec(nx=20, nz=20, dx=10.0, dz=10.0)
    sh = g.shape
    m = ElasticModel(grid=g, vp=np.full(sh, 2000.0, np.float32), vs=np.full(sh, 1000.0, np.float32),
                     rho=np.full(sh, 2000.0, np.float32), qp=np.full(sh, 50.0, np.float32),
                     qs=np.full(sh, 50.0, np.float32))
    with pytest.raises(SolverError):
        build_propagator(m, PropagationSpec(dt=1e-3, nt=10), engine="acoustic")


def test_float64_wavefields_are_rejected():
    from ertm_b200 import SolverError
    from ertm_b200.propagation import AcousticPropagator, PropagationSpec
    from ertm_b200.types import ElasticModel, GridSpec
    g = GridSpec(nx=20, nz=20, dx=10.0, dz=10.0)
    sh = g.shape
    m = ElasticModel(grid=g, vp=np.full(sh, 2000.0, np.float32), vs=np.full(sh, 1000.0, np.float32),
                     rho=np.full(sh, 2000.0, np.float32), qp=np.full(sh, 50.0, np.float32),
                     qs=np.full(sh, 50.0, np.float32))
    with pytest.raises(SolverError):
        AcousticPropagator(m, PropagationSpec(dt=1e-3, nt=10, dtype="float64"))


def test_serving_fails_loudly_without_a_device():
    """No GPU: the serving loop fails every submitted job instead of running
    anything on the host."""
    import types as _t

    from ertm_b200.serving import RTMServer, ServeJob, percentile
    job = ServeJob(shots=[], model=_t.SimpleNamespace(), imager=_t.SimpleNamespace(
        config=_t.SimpleNamespace(mode="pp")))
    srv = RTMServer()
    fut = srv.submit(job)
    srv.start()
    with pytest.raises(Exception):
        fut.result(timeout=60)
    srv.stop(timeout=60)
    assert percentile([1.0, 2.0, 3.0, 4.0], 50) == 2.5 and percentile([], 99) is None


def test_migrator_pool_reuses_and_rebuilds(monkeypatch):
    """Pool bookkeeping with a stand-in migrator (no device): pairs are
    handed out in order per group, reused by the next call, trimmed to the
    call's shot count, dropped for models the call does not use, and rebuilt
    when the material arrays or the solver settings change."""
    from ertm_b200 import ImagingConfig, RTMImager, SolverConfig
    from ertm_b200 import imaging
    from ertm_b200.types import ElasticModel, GridSpec

    built = []

    class Stub:
        def __init__(self, imager, model):
            self.model = model
            built.append(self)

    monkeypatch.setattr(imaging, "ShotMigrator", Stub)
    g = GridSpec(nx=8, nz=6, dx=5.0, dz=5.0)

    def model(v):
        a = np.full(g.shape, v, np.float32)
        return ElasticModel(grid=g, vp=a, vs=a / 2, rho=a.copy(), qp=a.copy(), qs=a.copy())

    imager = RTMImager(ImagingConfig(), SolverConfig(engine="acoustic"))
    pool = imaging.MigratorPool(imager)
    m1, m2 = model(2000.0), model(2500.0)
    pool.begin([m1, m1, m2])
    t: dict = {}
    a = [pool.take(m1, t), pool.take(m1, t), pool.take(m2, t)]
    assert len(built) == 3 and a[0] is not a[1]
    t = {}                                        # the next group of the same call reuses them
    assert pool.take(m1, t) is a[0] and pool.take(m1, t) is a[1] and len(built) == 3
    pool.begin([m1])                              # next call: one shot of m1 -> m2 dropped, m1 trimmed to one
    assert pool.take(m1, {}) is a[0] and len(built) == 3
    assert list(pool._entries) == [id(m1)] and len(pool._entries[id(m1)][2]) == 1
    m1.vp[2, 3] += 1.0                            # changed in place: stale
    pool.begin([m1])
    assert pool.take(m1, {}) is not a[0] and len(built) == 4
    imager.solver_config = dataclasses.replace(imager.solver_config, order=4)   # new settings: stale
    pool.begin([m1])
    pool.take(m1, {})
    assert len(built) == 5
    pool.begin([m1])                              # unchanged: kept
    pool.take(m1, {})
    assert len(built) == 5
    pool.clear()
    assert pool._entries == {}
