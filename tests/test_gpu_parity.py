"""CUDA path vs the reference: golden vectors and the CPU oracle.

Fields, CPML memories, shot records, image fields and migrated images of all
three engines are compared bit for bit: the kernels reproduce the
reference's float32 operation order, and the FFT low-pass (compensated
viscoacoustic stabilisation, image post-processing) reproduces numpy.fft's
arithmetic.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from helpers import (MIGRATE_CASES, PROPAGATION_CASES, imaging_from, load, model_from, q_from,
                     q_options_for_migrate, receivers_from, rel_l2, solver_from, source_from)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    import ertm_b200
    from ertm_b200 import _lib
    _lib.lib()  # fails loudly without the library or a B200
    return ertm_b200


def _product_propagation(eb, fx):
    from ertm_b200.propagation import PropagationSpec, QOptions, build_propagator
    meta = fx["meta"]
    dt, nt, order, npml = fx["spec"]
    spec = PropagationSpec(dt=float(dt), nt=int(nt), order=int(order), npml=int(npml), dtype="float32",
                           boundary=meta["boundary"])
    q = QOptions(**meta["q"]) if meta["q"] else None
    prop = build_propagator(model_from(fx), spec, engine=meta["engine"], q_options=q)
    prop.set_source(source_from(fx, meta["mechanism"]))
    prop.set_receivers(receivers_from(fx))
    names = meta["names"]
    rec = {n: np.zeros((int(nt), len(fx["rx"])), np.float32) for n in names}
    for t in range(int(nt)):
        if meta["inject_every"] and t % meta["inject_every"] == 0:
            for n in names:
                prop.inject(n, fx["inj_values"][t])
        prop.step(float(fx["wavelet"][t]))
        s = prop.sample(tuple(names))
        for n in names:
            rec[n][t] = s[n]
    return prop, rec


@pytest.mark.parametrize("case", PROPAGATION_CASES)
def test_propagation_matches_reference_golden(eb, case):
    fx = load(case)
    prop, rec = _product_propagation(eb, fx)
    st = prop.state()
    for k, v in st.items():
        key = f"state_{k.replace(':', '_')}"
        assert key in fx, key
        assert np.array_equal(v, fx[key]), (case, k, rel_l2(v, fx[key]))
    for n, r in rec.items():
        assert np.array_equal(r, fx[f"rec_{n}"]), (case, n, rel_l2(r, fx[f"rec_{n}"]))
    assert prop.state_bytes() == fx["meta"]["state_bytes"]
    if fx["meta"]["engine"] == "elastic":
        for sep in ("stress", "divcurl"):
            for k, v in prop.image_fields(sep).items():
                assert np.array_equal(v, fx[f"img_{sep}_{k}"]), (case, sep, k)
    if fx["meta"]["engine"] == "viscoacoustic":
        qs = prop.quality_summary
        assert qs["clipped"] == int(fx["clipped"])
        assert qs["lowpass_steps"] == int(fx["lowpass_steps"])


@pytest.mark.parametrize("case", MIGRATE_CASES)
def test_migrate_matches_reference_golden(eb, case):
    from ertm_b200 import ImagingConfig, QConfig, RTMImager, SolverConfig
    from ertm_b200.types import ReceiverSpec, ShotRecord, SourceSpec
    fx = load(case)
    meta = fx["meta"]
    comps = {k[len("shot_"):]: v for k, v in fx.items() if k.startswith("shot_") and k != "shot_dt"}
    src = source_from(fx)
    rec = receivers_from(fx)
    primary = comps[meta["components"][0]]
    shot = ShotRecord(data=primary, dt=float(fx["shot_dt"]), t=np.arange(primary.shape[0]) * float(fx["shot_dt"]),
                      receivers=ReceiverSpec(x=rec.x, z=rec.z),
                      source=SourceSpec(x=src.x, z=src.z, f0=src.f0, delay=src.delay), components=comps)
    imaging = ImagingConfig(mode=meta["mode"], condition=meta["condition"], separation=meta["separation"],
                            receiver_normalization=meta["receiver_normalization"], laplacian=True,
                            lowpass_fraction=meta["lowpass"], checkpoint_mb=meta["checkpoint_mb"])
    solver = SolverConfig(nt=meta["nt"], dt=meta["dt"], order=8, boundary=meta["boundary"], dtype="float32",
                          engine=meta["engine"], npml=12)
    q = QConfig(**meta["q"]) if meta["q"] else None
    img = RTMImager(imaging, solver, q).migrate(shot, model_from_types(fx))
    assert img.meta["checkpoints"]["interval"] == meta["checkpoints"]["interval"]
    assert img.meta["checkpoints"]["n_states"] == meta["checkpoints"]["n_states"]
    assert img.meta["start_step"] == meta["start_step"]
    assert np.array_equal(img.image, fx["image"]), (case, rel_l2(img.image, fx["image"]))


def model_from_types(fx):
    from ertm_b200.types import ElasticModel, GridSpec
    m = model_from(fx)
    g = m.grid
    return ElasticModel(grid=GridSpec(nx=g.nx, nz=g.nz, dx=g.dx, dz=g.dz, x0=g.x0, z0=g.z0),
                        vp=m.vp, vs=m.vs, rho=m.rho, qp=m.qp, qs=m.qs)


def test_migrate_pp_ps_in_one_pass_equals_separate_runs(eb):
    """One forward/replay/backward pass imaging PP and PS gives the single-mode images."""
    from ertm_b200 import ImagingConfig, RTMImager, SolverConfig
    from ertm_b200.types import ReceiverSpec, ShotRecord, SourceSpec
    fx = load("mig_elastic_pp_divcurl")
    meta = fx["meta"]
    comps = {k[len("shot_"):]: v for k, v in fx.items() if k.startswith("shot_") and k != "shot_dt"}
    src = source_from(fx)
    rec = receivers_from(fx)
    primary = comps[meta["components"][0]]
    shot = ShotRecord(data=primary, dt=float(fx["shot_dt"]), t=np.arange(primary.shape[0]) * float(fx["shot_dt"]),
                      receivers=ReceiverSpec(x=rec.x, z=rec.z),
                      source=SourceSpec(x=src.x, z=src.z, f0=src.f0, delay=src.delay), components=comps)
    solver = SolverConfig(nt=meta["nt"], dt=meta["dt"], order=8, boundary=meta["boundary"], engine="elastic",
                          npml=12)
    model = model_from_types(fx)
    both = RTMImager(ImagingConfig(mode="pp", condition="normalized", checkpoint_mb=1.0), solver).migrate_modes(
        shot, model, modes=("pp", "ps"))
    for res in both:
        single = RTMImager(ImagingConfig(mode=res.mode, condition="normalized", checkpoint_mb=1.0),
                           solver).migrate(shot, model)
        assert np.array_equal(res.image, single.image), res.mode


def test_checkpoint_replay_is_bit_exact(eb):
    """Mirror of the reference KAT (tests/test_rtm.py:188-214) on the device."""
    from ertm_b200.propagation import AcousticPropagator, PropagationSpec, source_wavelet
    from ertm_b200.types import ElasticModel, GridSpec, SourceSpec
    g = GridSpec(nx=61, nz=51, dx=10.0, dz=10.0)
    sh = g.shape
    model = ElasticModel(grid=g, vp=np.full(sh, 3000.0, np.float32), vs=np.full(sh, 1700.0, np.float32),
                         rho=np.full(sh, 2400.0, np.float32), qp=np.full(sh, 100.0, np.float32),
                         qs=np.full(sh, 50.0, np.float32))
    spec = PropagationSpec(dt=5e-4, nt=80, order=8, npml=8, dtype="float32", boundary="cpml")
    src = SourceSpec(x=300.0, z=250.0, f0=20.0, delay=0.03)
    w = source_wavelet(src, spec.dt, spec.nt)
    ref = AcousticPropagator(model, spec)
    ref.set_source(src)
    for t in range(60):
        ref.step(float(w[t]))
    rep = AcousticPropagator(model, spec)
    rep.set_source(src)
    rep.step(float(w[0]))
    rep.load_state(rep.state())
    for t in range(1, 60):
        rep.step(float(w[t]))
    assert np.array_equal(rep.p, ref.p)
    expected = sum(getattr(rep, n).nbytes for n in ("p", "vx", "vz")) + rep.pml.memory_bytes()
    assert rep.state_bytes() == expected


@pytest.mark.parametrize("engine,boundary,order", [("acoustic", "cpml", 8), ("acoustic", "free", 4),
                                                   ("elastic", "free", 8), ("elastic", "cpml", 6),
                                                   ("viscoacoustic", "cpml", 8), ("acoustic", "none", 2)])
def test_forward_record_matches_oracle_on_seeded_models(eb, engine, boundary, order):
    """Seeded layered model, non-square grid, all stencil orders: GPU == oracle."""
    from ertm_b200.propagation import PropagationSpec, QOptions, run_forward
    rng = np.random.default_rng(7)
    nz, nx = 53, 71
    vp = rng.uniform(2000.0, 3000.0, size=(nz, nx)).astype(np.float32)
    model = model_from({"m_vp": vp, "m_vs": (vp / 1.9).astype(np.float32),
                        "m_rho": rng.uniform(1800, 2400, (nz, nx)).astype(np.float32),
                        "m_qp": np.where(np.arange(nz)[:, None] < 25, 40.0, 90.0).repeat(nx, 1).astype(np.float32),
                        "m_qs": np.full((nz, nx), 30.0, np.float32),
                        "m_grid": np.array([nx, nz, 8.0, 6.0, 0.0, 0.0])})
    dt = 0.8 * orc.cfl_dt(float(vp.max()), 8.0, 6.0, order, 0.5)
    spec = PropagationSpec(dt=dt, nt=120, order=order, npml=10, boundary=boundary)
    src = source_from({"src": np.array([260.0, 50.0, 30.0, 0.03, 1.0])})
    rcv = receivers_from({"rx": rng.uniform(-10, 570, 23), "rz": rng.uniform(0, 320, 23)})
    comps = ("p", "vx", "vz") if engine != "elastic" else ("p", "vx", "vz", "sxz")
    q = QOptions(enabled=True, f_ref=30.0) if engine == "viscoacoustic" else None
    got = run_forward(model, src, rcv, spec, engine=engine, components=comps, q_options=q)
    ospec = orc.Spec(dt=dt, nt=120, order=order, npml=10, boundary=boundary)
    want = orc.run_forward(model, src, rcv, ospec, engine=engine, components=comps, q=q)
    for n in comps:
        assert np.array_equal(got[n], want[n]), (n, rel_l2(got[n], want[n]))


def test_stack_images_matches_reference_golden(eb):
    from ertm_b200.stacking import stack_arrays
    fx = load("stack")
    assert np.array_equal(stack_arrays(list(fx["images"])), fx["stacked"])


def test_kahan_accumulation_close_to_fp64(eb):
    """Form (a): Kahan-compensated FP32 imaging sums vs the FP64 accumulators."""
    from ertm_b200 import ImagingConfig, RTMImager, SolverConfig
    from ertm_b200.types import ReceiverSpec, ShotRecord, SourceSpec
    fx = load("mig_acoustic_norm_rn")
    meta = fx["meta"]
    src, rec = source_from(fx), receivers_from(fx)
    data = fx["shot_p"]
    shot = ShotRecord(data=data, dt=float(fx["shot_dt"]), t=np.arange(data.shape[0]) * float(fx["shot_dt"]),
                      receivers=ReceiverSpec(x=rec.x, z=rec.z),
                      source=SourceSpec(x=src.x, z=src.z, f0=src.f0, delay=src.delay), components={"p": data})
    solver = SolverConfig(nt=meta["nt"], dt=meta["dt"], boundary=meta["boundary"], engine="acoustic", npml=12)
    imaging = ImagingConfig(condition="normalized", receiver_normalization=True, checkpoint_mb=1.0)
    a = RTMImager(imaging, solver).migrate(shot, model_from_types(fx))
    b = RTMImager(imaging, solver, accumulation="kahan").migrate(shot, model_from_types(fx))
    assert rel_l2(b.image, a.image) < 1e-5


@pytest.fixture
def split_always(eb):
    """Interior tiles in launches of their own even on small grids."""
    from ertm_b200 import _lib
    _lib.check(_lib.lib().ertm_set_tile_split(2), "split")
    yield
    _lib.check(_lib.lib().ertm_set_tile_split(0), "split")


@pytest.mark.parametrize("march,march_stress", [(0, 0), (4, 0), (8, 0), (4, 1)])
@pytest.mark.parametrize("frame_rows", [0, 8])
@pytest.mark.parametrize("tma", [1, 0])
@pytest.mark.parametrize("engine,boundary,mechanism,tile_rows", [
    ("acoustic", "cpml", "explosive", 16), ("acoustic", "free", "explosive", 8),
    ("elastic", "free", "explosive", 16), ("elastic", "cpml", "force_z", 8), ("elastic", "free", "shear", 32),
    ("viscoacoustic", "cpml", "explosive", 16)])
def test_interior_and_boundary_launches_match_oracle(eb, split_always, engine, boundary, mechanism, tile_rows, tma,
                                                     frame_rows, march, march_stress):
    """Interior tiles and the boundary frame in separate launches (the source
    node's tile, inside the interior rectangle, goes with the frame, as one
    tile or as several lower frame tiles), interior tiles staged by TMA or by
    cp.async: GPU == oracle on a grid with an interior rectangle of several
    tiles."""
    from ertm_b200 import _lib
    from ertm_b200.propagation import PropagationSpec, QOptions, run_forward
    _lib.check(_lib.lib().ertm_set_tile_rows(tile_rows), "tile rows")
    _lib.check(_lib.lib().ertm_set_tma(tma), "tma")
    _lib.check(_lib.lib().ertm_set_frame_rows(frame_rows), "frame rows")
    _lib.check(_lib.lib().ertm_set_march(march), "march")
    _lib.check(_lib.lib().ertm_set_march_stress(march_stress), "march stress")
    try:
        rng = np.random.default_rng(11)
        nz, nx = 150, 200
        vp = rng.uniform(2000.0, 3000.0, size=(nz, nx)).astype(np.float32)
        model = model_from({"m_vp": vp, "m_vs": (vp / 1.9).astype(np.float32),
                            "m_rho": rng.uniform(1800, 2400, (nz, nx)).astype(np.float32),
                            "m_qp": np.where(np.arange(nz)[:, None] < 70, 40.0, 90.0).repeat(nx, 1).astype(np.float32),
                            "m_qs": np.full((nz, nx), 30.0, np.float32),
                            "m_grid": np.array([nx, nz, 5.0, 5.0, 0.0, 0.0])})
        dt = 0.8 * orc.cfl_dt(float(vp.max()), 5.0, 5.0, 8, 0.5)
        spec = PropagationSpec(dt=dt, nt=90, order=8, npml=12, boundary=boundary)
        src = source_from({"src": np.array([502.0, 371.0, 40.0, 0.02, 1.0])}, mechanism)
        rcv = receivers_from({"rx": rng.uniform(0, 995, 31), "rz": rng.uniform(0, 745, 31)})
        comps = ("p", "vx", "vz") if engine != "elastic" else ("p", "vx", "vz", "sxz")
        q = QOptions(enabled=True, f_ref=30.0) if engine == "viscoacoustic" else None
        got = run_forward(model, src, rcv, spec, engine=engine, components=comps, q_options=q)
        ospec = orc.Spec(dt=dt, nt=90, order=8, npml=12, boundary=boundary)
        want = orc.run_forward(model, src, rcv, ospec, engine=engine, components=comps, q=q)
    finally:
        _lib.check(_lib.lib().ertm_set_tile_rows(0), "tile rows")
        _lib.check(_lib.lib().ertm_set_tma(0), "tma")
        _lib.check(_lib.lib().ertm_set_frame_rows(0), "frame rows")
        _lib.check(_lib.lib().ertm_set_march(4), "march")
        _lib.check(_lib.lib().ertm_set_march_stress(0), "march stress")
    assert _lib.lib().ertm_stage_timeouts() == 0
    for n in comps:
        assert np.array_equal(got[n], want[n]), (n, rel_l2(got[n], want[n]))


def test_batched_images_equal_with_and_without_split_launches(eb):
    """The batched migration gives the same images whether interior tiles run
    in launches of their own or with the boundary tiles, and whether a tick's
    works run in one stream lane or two."""
    from ertm_b200 import ImagingConfig, RTMImager, SolverConfig, _lib
    from ertm_b200.batch import BatchMigrator
    from ertm_b200.propagation import PropagationSpec, forward_shot
    from ertm_b200.types import ElasticModel, GridSpec, ReceiverSpec, SourceSpec
    rng = np.random.default_rng(5)
    g = GridSpec(nx=180, nz=140, dx=5.0, dz=5.0)
    vp = (2200.0 + 900.0 * (np.arange(g.nz)[:, None] > 70) + rng.uniform(0, 60, g.shape)).astype(np.float32)
    model = ElasticModel(grid=g, vp=vp, vs=(vp / 1.8).astype(np.float32), rho=np.full(g.shape, 2100.0, np.float32),
                         qp=np.full(g.shape, 80.0, np.float32), qs=np.full(g.shape, 40.0, np.float32))
    x = np.arange(0.0, 895.0, 20.0)
    rec = ReceiverSpec(x=x, z=np.full_like(x, 10.0))
    shots = [forward_shot(model, SourceSpec(x=300.0 + 150.0 * k, z=10.0, f0=30.0, delay=0.03), rec,
                          PropagationSpec(dt=4e-4, nt=260, npml=20, boundary="free"), engine="elastic",
                          components=("vz", "p")) for k in range(3)]
    imager = RTMImager(ImagingConfig(condition="normalized", checkpoint_mb=2.0),
                       SolverConfig(nt=260, dt=4e-4, boundary="free", engine="elastic"))
    out = {}
    cases = ((1, 1, 0, 0, 0), (2, 1, 0, 0, 0), (2, 2, 0, 0, 0), (1, 2, 0, 0, 0), (2, 2, 1, 0, 0), (1, 2, 1, 0, 0),
             (2, 2, 0, 32, 8), (2, 1, 0, 32, 16), (2, 2, 1, 16, 8), (2, 4, 0, 0, 0), (1, 4, 1, 32, 0),
             (2, 2, 0, 32, 0, 8), (2, 1, 0, 32, 16, 2), (2, 2, 0, 32, 0, 0), (2, 2, 0, 32, 0, 4, 1))
    for mode, lanes, assign, rows, frame_rows, *rest in cases:
        _lib.check(_lib.lib().ertm_set_tile_split(mode), "split")
        _lib.check(_lib.lib().ertm_set_tick_lanes(lanes), "lanes")
        _lib.check(_lib.lib().ertm_set_lane_assign(assign), "lane assignment")
        _lib.check(_lib.lib().ertm_set_tile_rows(rows), "tile rows")
        _lib.check(_lib.lib().ertm_set_frame_rows(frame_rows), "frame rows")
        _lib.check(_lib.lib().ertm_set_march(rest[0] if rest else 4), "march")
        _lib.check(_lib.lib().ertm_set_march_stress(rest[1] if len(rest) > 1 else 0), "march stress")
        try:
            out[(mode, lanes, assign, rows, frame_rows, *rest)] = BatchMigrator(imager).migrate_shots(
                shots, model, modes=("pp", "ps"))
        finally:
            _lib.check(_lib.lib().ertm_set_tile_split(0), "split")
            _lib.check(_lib.lib().ertm_set_tick_lanes(0), "lanes")
            _lib.check(_lib.lib().ertm_set_lane_assign(0), "lane assignment")
            _lib.check(_lib.lib().ertm_set_tile_rows(0), "tile rows")
            _lib.check(_lib.lib().ertm_set_frame_rows(0), "frame rows")
            _lib.check(_lib.lib().ertm_set_march(4), "march")
            _lib.check(_lib.lib().ertm_set_march_stress(0), "march stress")
    for key in cases[1:]:
        for a, b in zip(out[cases[0]], out[key]):
            for x1, x2 in zip(a, b):
                assert np.array_equal(x1.image, x2.image), (key, x1.mode)


def test_autotuned_batch_equals_untuned(eb):
    """The online autotuner switches launch shapes between the first ticks of
    a batch; the images equal those of a run with tuning off."""
    from ertm_b200 import ImagingConfig, RTMImager, SolverConfig, _lib
    from ertm_b200.batch import BatchMigrator
    from ertm_b200.propagation import PropagationSpec, forward_shot
    from ertm_b200.types import ElasticModel, GridSpec, ReceiverSpec, SourceSpec
    rng = np.random.default_rng(9)
    g = GridSpec(nx=420, nz=300, dx=5.0, dz=5.0)
    vp = (2400.0 + 700.0 * (np.arange(g.nz)[:, None] > 150) + rng.uniform(0, 50, g.shape)).astype(np.float32)
    model = ElasticModel(grid=g, vp=vp, vs=(vp / 1.8).astype(np.float32), rho=np.full(g.shape, 2100.0, np.float32),
                         qp=np.full(g.shape, 80.0, np.float32), qs=np.full(g.shape, 40.0, np.float32))
    x = np.arange(0.0, 2095.0, 40.0)
    rec = ReceiverSpec(x=x, z=np.full_like(x, 10.0))
    shots = [forward_shot(model, SourceSpec(x=500.0 + 400.0 * k, z=10.0, f0=25.0, delay=0.04), rec,
                          PropagationSpec(dt=4e-4, nt=240, npml=20, boundary="free"), engine="elastic",
                          components=("vz", "p")) for k in range(3)]
    imager = RTMImager(ImagingConfig(condition="normalized", checkpoint_mb=8.0),
                       SolverConfig(nt=240, dt=4e-4, boundary="free", engine="elastic"))
    L = _lib.lib()
    out = {}
    try:
        for mode in (0, -1, 1):
            _lib.check(L.ertm_set_autotune(mode), "autotune")
            out[mode] = BatchMigrator(imager).migrate_shots(shots, model, modes=("pp", "ps"))
    finally:
        _lib.check(L.ertm_set_autotune(1), "autotune")
    for mode in (-1, 1):
        for a, b in zip(out[0], out[mode]):
            for x1, x2 in zip(a, b):
                assert np.array_equal(x1.image, x2.image), (mode, x1.mode)
