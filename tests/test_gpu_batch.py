"""Form (b): batched migration equals the plain one-shot path bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import MIGRATE_CASES, load, rel_l2

pytestmark = pytest.mark.gpu


def _inputs(case: str):
    from ertm_b200 import ImagingConfig, QConfig, SolverConfig
    from ertm_b200.types import ElasticModel, GridSpec, ReceiverSpec, ShotRecord, SourceSpec
    fx = load(case)
    meta = fx["meta"]
    nx, nz, dx, dz, x0, z0 = fx["m_grid"]
    g = GridSpec(nx=int(nx), nz=int(nz), dx=float(dx), dz=float(dz))
    model = ElasticModel(grid=g, vp=fx["m_vp"], vs=fx["m_vs"], rho=fx["m_rho"], qp=fx["m_qp"], qs=fx["m_qs"])
    comps = {k[len("shot_"):]: v for k, v in fx.items() if k.startswith("shot_") and k != "shot_dt"}
    primary = comps[meta["components"][0]]
    rec = ReceiverSpec(x=fx["rx"], z=fx["rz"])
    x, z, f0, delay, _ = fx["src"]
    shots = []
    for shift in (0.0, -60.0, 90.0):
        src = SourceSpec(x=float(x) + shift, z=float(z), f0=float(f0), delay=float(delay))
        shots.append(ShotRecord(data=primary, dt=float(fx["shot_dt"]), t=np.arange(primary.shape[0]) * fx["shot_dt"],
                                receivers=rec, source=src, components=comps))
    imaging = ImagingConfig(mode=meta["mode"], condition=meta["condition"], separation=meta["separation"],
                            receiver_normalization=meta["receiver_normalization"], laplacian=True,
                            lowpass_fraction=meta["lowpass"], checkpoint_mb=meta["checkpoint_mb"])
    solver = SolverConfig(nt=meta["nt"], dt=meta["dt"], order=8, boundary=meta["boundary"], engine=meta["engine"],
                          npml=12)
    q = QConfig(**meta["q"]) if meta["q"] else None
    return fx, model, shots, imaging, solver, q


@pytest.mark.parametrize("case", MIGRATE_CASES)
def test_batch_equals_plain(case):
    from ertm_b200 import RTMImager
    from ertm_b200.batch import BatchMigrator
    fx, model, shots, imaging, solver, q = _inputs(case)
    imager = RTMImager(imaging, solver, q)
    modes = ("pp", "ps") if fx["meta"]["engine"] == "elastic" else ("pp",)
    batched = BatchMigrator(imager).migrate_shots(shots, model, modes=modes)
    for shot, res in zip(shots, batched):
        plain = imager.migrate_modes(shot, model, modes=modes)
        for a, b in zip(res, plain):
            assert a.mode == b.mode
            assert np.array_equal(a.image, b.image), (case, a.mode, rel_l2(a.image, b.image))
    if fx["meta"]["mode"] == "pp":
        assert rel_l2(batched[0][0].image, fx["image"]) < 1e-6


def test_batch_mixed_grids_and_lengths():
    """Uneven batch: two models of different size, shots of different length."""
    from ertm_b200 import ImagingConfig, RTMImager, SolverConfig
    from ertm_b200.batch import BatchMigrator
    from ertm_b200.propagation import PropagationSpec, forward_shot
    from ertm_b200.types import ElasticModel, GridSpec, ReceiverSpec, SourceSpec
    rng = np.random.default_rng(3)
    models = []
    for nx, nz in ((57, 41), (83, 49)):
        g = GridSpec(nx=nx, nz=nz, dx=10.0, dz=10.0)
        vp = (2000.0 + 800.0 * (np.arange(nz)[:, None] > nz // 2) + rng.uniform(0, 50, (nz, nx))).astype(np.float32)
        models.append(ElasticModel(grid=g, vp=vp, vs=(vp / 1.8).astype(np.float32), rho=np.full(g.shape, 2000.0, np.float32),
                                   qp=np.full(g.shape, 80.0, np.float32), qs=np.full(g.shape, 40.0, np.float32)))
    shots, mlist, wavelets = [], [], []
    for k, (m, nt) in enumerate([(models[0], 240), (models[1], 300), (models[0], 180), (models[1], 260)]):
        src = SourceSpec(x=200.0 + 40.0 * k, z=20.0, f0=25.0, delay=0.04)
        x = np.linspace(0.0, (m.grid.nx - 1) * 10.0, 20)
        rec = ReceiverSpec(x=x, z=np.full_like(x, 20.0))
        shot = forward_shot(m, src, rec, PropagationSpec(dt=8e-4, nt=nt, npml=10, boundary="free"))
        shots.append(shot)
        mlist.append(m)
        from ertm_b200.propagation import source_wavelet
        wavelets.append(source_wavelet(src, 8e-4, 300))
    imager = RTMImager(ImagingConfig(condition="normalized", checkpoint_mb=1.0),
                       SolverConfig(nt=300, dt=8e-4, boundary="free", engine="acoustic", npml=10))
    batched = BatchMigrator(imager).migrate_shots(shots, mlist, wavelets=[w[: s.data.shape[0]] for w, s in
                                                                         zip(wavelets, shots)])
    for shot, m, res, w in zip(shots, mlist, batched, wavelets):
        plain = imager.migrate(shot, m, wavelet=w[: shot.data.shape[0]])
        assert np.array_equal(res[0].image, plain.image)


def test_batch_memory_grouping_gives_same_images():
    """A tiny budget forces one shot per group; images are unchanged."""
    from ertm_b200 import RTMImager
    from ertm_b200.batch import BatchMigrator
    fx, model, shots, imaging, solver, q = _inputs("mig_acoustic_zerolag")
    imager = RTMImager(imaging, solver, q)
    a = BatchMigrator(imager).migrate_shots(shots, model)
    b = BatchMigrator(imager, memory_budget=1).migrate_shots(shots, model)
    for x, y in zip(a, b):
        assert np.array_equal(x[0].image, y[0].image)


def test_pooled_pairs_give_fresh_results():
    """A BatchMigrator and an RTMImager reuse their propagator pairs between
    calls; the images equal those of freshly built pairs bit for bit, and a
    model changed in place gets new pairs."""
    from ertm_b200 import RTMImager
    from ertm_b200.batch import BatchMigrator
    fx, model, shots, imaging, solver, q = _inputs("mig_visco_comp")
    imager = RTMImager(imaging, solver, q)
    bm = BatchMigrator(imager)
    first = bm.migrate_shots(shots, model)
    pairs = list(bm._pool._entries[id(model)][2])
    again = bm.migrate_shots(shots[::-1], model)
    assert [p is q_ for p, q_ in zip(bm._pool._entries[id(model)][2], pairs)] == [True] * len(pairs)
    for a, b in zip(first, again[::-1]):
        assert np.array_equal(a[0].image, b[0].image)
    # one pair serves every group when the budget forces one shot per group
    small = BatchMigrator(imager, memory_budget=1)
    one = small.migrate_shots(shots, model)
    assert len(small._pool._entries[id(model)][2]) == 1
    for a, b in zip(first, one):
        assert np.array_equal(a[0].image, b[0].image)
    # the imager's single-shot path keeps one pair for the next call
    p1 = imager.migrate(shots[1], model)
    kept = imager._pool._entries[id(model)][2][0]
    p2 = imager.migrate(shots[1], model)
    assert imager._pool._entries[id(model)][2][0] is kept
    assert np.array_equal(p1.image, p2.image) and np.array_equal(p1.image, first[1][0].image)
    # a model changed in place: new pairs, images of the changed model
    vp0 = model.vp.copy()
    try:
        model.vp[model.vp.shape[0] // 2:, :] *= np.float32(0.97)     # slower: stays stable
        changed = bm.migrate_shots(shots, model)
        assert all(p is not q_ for p, q_ in zip(bm._pool._entries[id(model)][2], pairs))
        fresh = BatchMigrator(RTMImager(imaging, solver, q)).migrate_shots(shots, model)
        for a, b in zip(changed, fresh):
            assert np.array_equal(a[0].image, b[0].image)
        assert not np.array_equal(changed[0][0].image, first[0][0].image)
    finally:
        model.vp[...] = vp0
