"""Generate the golden vectors by running the reference ERTM code itself.

Run in a container that holds the reference checkout (read-only):

    python tests/golden/make_golden.py [/path/to/reference]

It imports the reference's own ``ertm`` package (numerics, propagation,
imaging, viscoelastic, preprocess, qcomp, data; pipeline.stack_images
restated inline because ``ertm.pipeline`` needs matplotlib), feeds it small
seeded inputs and writes the inputs and outputs to ``tests/golden/*.npz``;
the ``store`` case also keeps the three .npz files the reference's
NumpyDataStore wrote, under ``tests/golden/store/``.  Cases by name:

    python tests/golden/make_golden.py /path/to/reference qcomp store  The committed fixtures
pin both the CPU oracle and the CUDA path; nothing at test time reads the
reference tree.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
sys.path.insert(0, str(REF))

from ertm import numerics as num  # noqa: E402
from ertm import viscoelastic as ve  # noqa: E402
from ertm.config import ImagingConfig, QConfig, SolverConfig  # noqa: E402
from ertm.imaging import RTMImager  # noqa: E402
from ertm.propagation import (  # noqa: E402
    PropagationSpec,
    QOptions,
    build_propagator,
    forward_shot,
    source_wavelet,
)
from ertm.types import ElasticModel, GridSpec, ReceiverSpec, SourceSpec  # noqa: E402


def layered_model(nx: int, nz: int, dx: float, seed: int, *, q_layers=(60.0, 30.0, 100.0)) -> ElasticModel:
    """Three dipping layers plus a lens; float32 arrays like the reference builders."""
    rng = np.random.default_rng(seed)
    grid = GridSpec(nx=nx, nz=nz, dx=dx, dz=dx)
    x = np.arange(nx) * dx
    z = np.arange(nz) * dx
    xx, zz = np.meshgrid(x, z)
    t1 = nz * dx * 0.35 + 0.1 * (xx - x.mean())
    t2 = nz * dx * 0.65 - 0.05 * (xx - x.mean())
    vp = np.where(zz < t1, 2000.0, np.where(zz < t2, 2600.0, 3200.0))
    vp = vp + rng.uniform(-50.0, 50.0, size=vp.shape)
    lens = (xx - x.mean()) ** 2 / (0.15 * nx * dx) ** 2 + (zz - 0.5 * nz * dx) ** 2 / (0.08 * nz * dx) ** 2 < 1
    vp = np.where(lens, 1800.0, vp).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = (310.0 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    qp = np.where(zz < t1, q_layers[0], np.where(zz < t2, q_layers[1], q_layers[2])).astype(np.float32)
    qs = (qp * 0.5).astype(np.float32)
    return ElasticModel(grid=grid, vp=vp, vs=vs, rho=rho, qp=qp, qs=qs)


def model_arrays(prefix: str, m: ElasticModel) -> dict[str, np.ndarray]:
    g = m.grid
    return {
        f"{prefix}vp": m.vp, f"{prefix}vs": m.vs, f"{prefix}rho": m.rho,
        f"{prefix}qp": m.qp, f"{prefix}qs": m.qs,
        f"{prefix}grid": np.array([g.nx, g.nz, g.dx, g.dz, g.x0, g.z0], dtype=np.float64),
    }


def receivers_line(x0: float, x1: float, n: int, z: float) -> ReceiverSpec:
    x = np.linspace(x0, x1, n)
    return ReceiverSpec(x=x, z=np.full_like(x, z), component="p")


def numerics_case() -> dict[str, np.ndarray]:
    rng = np.random.default_rng(11)
    out: dict[str, np.ndarray] = {}
    f = rng.normal(size=(23, 29)).astype(np.float32)
    out["deriv_in"] = f
    for order in (2, 4, 6, 8):
        c = num.staggered_coefficients(order)
        for axis in (0, 1):
            h = 7.5 if axis == 1 else 5.0
            out[f"dplus_o{order}_a{axis}"] = num.dplus(f, axis, c, h)
            out[f"dminus_o{order}_a{axis}"] = num.dminus(f, axis, c, h)
    for i, (length, h, npml, dt, vmax, sides, enabled) in enumerate([
        (61, 10.0, 20, 1e-3, 3000.0, (True, True), True),
        (41, 5.0, 40, 3e-4, 4500.0, (False, True), True),
        (30, 10.0, 8, 5e-4, 2500.0, (True, True), False),
    ]):
        ax = num.CPMLAxis(length, h, npml, dt, vmax, axis=1, alpha_max=2.0 * np.pi * 25.0,
                          sides=sides, enabled=enabled)
        out[f"cpml{i}_b"] = ax.b.ravel()
        out[f"cpml{i}_a"] = ax.a.ravel()
        out[f"cpml{i}_npml"] = np.array(ax.npml)
    out["cfl"] = np.array([num.cfl_dt(v, dx, dz, o, s) for v, dx, dz, o, s in [
        (3000.0, 10.0, 10.0, 8, 0.5), (4500.0, 5.0, 5.0, 8, 0.55), (4000.0, 5.0, 5.0, 4, 0.5)]])
    t = np.arange(300) * 1e-3
    out["ricker"] = num.ricker(t, 15.0, 0.08)
    img = rng.normal(size=(37, 45))
    out["img_in"] = img
    out["laplacian"] = num.laplacian(img, 10.0, 5.0)
    out["lowpass"] = num.lowpass_wavenumber(img, 10.0, 5.0, 0.85)
    zi = rng.uniform(-1.0, 24.0, size=40)
    xi = rng.uniform(-1.0, 30.0, size=40)
    out["bil_z"], out["bil_x"] = zi, xi
    out["bilinear"] = num.bilinear_sample(f, zi, xi)
    rec = rng.normal(size=(120, 5))
    out["resample_in"] = rec
    out["resample"] = num.resample_sinc(rec, 4e-4, 2.5e-4)
    return out


def gsls_case() -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    qs = [15.0, 25.0, 40.0, 60.0, 100.0, 200.0, 2e4]
    out["q"] = np.array(qs)
    for n in (1, 3):
        taus, deltas, errs, mref = [], [], [], []
        for q in qs:
            p = ve.fit_gsls(q, 30.0, n_mechanisms=n, band_ratio=1.5)
            tau = np.full(n, np.nan)
            dlt = np.full(n, np.nan)
            tau[: len(p.tau_sigma)] = p.tau_sigma
            dlt[: len(p.delta)] = p.delta
            taus.append(tau)
            deltas.append(dlt)
            errs.append(p.fit_error)
            mref.append(float(np.real(ve.normalized_modulus(p.tau_sigma, p.delta, [30.0])[0])))
        out[f"tau_n{n}"] = np.array(taus)
        out[f"delta_n{n}"] = np.array(deltas)
        out[f"err_n{n}"] = np.array(errs)
        out[f"mref_n{n}"] = np.array(mref)
    return out


def propagate_case(engine: str, boundary: str, *, nt: int, mechanism: str = "explosive",
                   q: QOptions | None = None, seed: int = 3, dtype: str = "float32",
                   inject_every: int = 0) -> dict[str, np.ndarray]:
    """Step a propagator, sample every step, optionally inject a seeded trace."""
    m = layered_model(47, 37, 10.0, seed)
    spec = PropagationSpec(dt=8e-4, nt=nt, order=8, npml=9, dtype=dtype, boundary=boundary)
    prop = build_propagator(m, spec, engine=engine, q_options=q)
    src = SourceSpec(x=233.0, z=40.0, f0=25.0, delay=0.04, mechanism=mechanism)
    prop.set_source(src)
    rx = np.array([13.0, 77.5, 140.0, 141.0, 205.0, 260.0, 300.0, 404.9, 460.0, -3.0])
    rz = np.array([20.0, 20.0, 22.5, 22.5, 75.0, 31.0, 300.0, 150.0, 355.0, 20.0])
    rec = ReceiverSpec(x=rx, z=rz)
    prop.set_receivers(rec)
    wave = source_wavelet(src, spec.dt, spec.nt)
    names = prop.components
    if engine == "elastic":
        names = ("p", "vx", "vz", "sxz")
    samples = {n: np.zeros((nt, rec.nrec), dtype=np.float32) for n in names}
    rng = np.random.default_rng(seed + 100)
    inj_values = rng.normal(size=(nt, rec.nrec)).astype(np.float32)
    for t in range(nt):
        if inject_every and t % inject_every == 0:
            for n in names:
                prop.inject(n, inj_values[t])
        prop.step(float(wave[t]))
        s = prop.sample(names)
        for n in names:
            samples[n][t] = s[n]
    out = model_arrays("m_", m)
    out.update({
        "spec": np.array([spec.dt, spec.nt, spec.order, spec.npml]),
        "src": np.array([src.x, src.z, src.f0, src.delay, src.amplitude]),
        "rx": rx, "rz": rz, "wavelet": wave, "inj_values": inj_values,
    })
    for k, v in prop.state().items():
        out[f"state_{k.replace(':', '_')}"] = np.asarray(v)
    for n in names:
        out[f"rec_{n}"] = samples[n]
    if engine == "elastic":
        for sep in ("stress", "divcurl"):
            for k, v in prop.image_fields(sep).items():
                out[f"img_{sep}_{k}"] = np.asarray(v)
    out["meta"] = np.array(json.dumps({
        "engine": engine, "boundary": boundary, "mechanism": mechanism, "dtype": dtype,
        "inject_every": inject_every, "names": list(names),
        "q": None if q is None else q.__dict__,
        "state_bytes": prop.state_bytes(),
    }))
    if engine == "viscoacoustic":
        out["k_relaxed"] = prop.k_relaxed
        out["relax_a"] = prop.a
        out["relax_b"] = prop.b
        out["clipped"] = np.array(getattr(prop, "_clipped", 0))
        out["lowpass_steps"] = np.array(getattr(prop, "_lowpass_steps", 0))
    return out


def migrate_case(engine: str, condition: str, *, boundary: str, mode: str = "pp",
                 separation: str = "divcurl", receiver_normalization: bool = False,
                 q: QConfig | None = None, nt: int = 260, seed: int = 5,
                 components: tuple[str, ...] | None = None, lowpass: float = 0.85,
                 checkpoint_mb: float = 1.0) -> dict[str, np.ndarray]:
    m = layered_model(51, 41, 10.0, seed)
    solver = SolverConfig(nt=nt, dt=8e-4, order=8, boundary=boundary, dtype="float32",
                          engine=engine, npml=12)
    spec = PropagationSpec.from_config(solver, m, npml=solver.npml)
    src = SourceSpec(x=250.0, z=20.0, f0=25.0, delay=0.04)
    rec = receivers_line(0.0, 500.0, 26, 20.0)
    qopt = None
    if engine == "viscoacoustic":
        qq = q or QConfig()
        qopt = QOptions(enabled=True, f_ref=qq.f_ref, n_mechanisms=qq.n_mechanisms,
                        band_ratio=qq.band_ratio, compensation=False, alpha_c=qq.alpha_c,
                        amplitude_cap=qq.amplitude_cap, lowpass_interval=qq.lowpass_interval,
                        f_max=qq.f_max, gain_budget_db=qq.gain_budget_db)
    shot = forward_shot(m, src, rec, spec, engine=engine, components=components, q_options=qopt)
    imaging = ImagingConfig(mode=mode, condition=condition, separation=separation,
                            receiver_normalization=receiver_normalization, laplacian=True,
                            lowpass_fraction=lowpass, checkpoint_mb=checkpoint_mb)
    imager = RTMImager(imaging, solver, q)
    image = imager.migrate(shot, m)
    out = model_arrays("m_", m)
    out.update({
        "src": np.array([src.x, src.z, src.f0, src.delay, src.amplitude]),
        "rx": rec.x, "rz": rec.z, "shot_dt": np.array(shot.dt),
        "image": image.image,
    })
    for k, v in shot.components.items():
        out[f"shot_{k}"] = v
    out["meta"] = np.array(json.dumps({
        "engine": engine, "condition": condition, "boundary": boundary, "mode": mode,
        "separation": separation, "receiver_normalization": receiver_normalization,
        "nt": nt, "dt": 8e-4, "lowpass": lowpass, "checkpoint_mb": checkpoint_mb,
        "components": list(shot.components), "q": None if q is None else q.__dict__,
        "checkpoints": image.meta["checkpoints"], "start_step": image.meta["start_step"],
        "npml": image.meta["npml"], "forward_npml": spec.npml,
    }))
    return out


def stack_case() -> dict[str, np.ndarray]:
    """pipeline.stack_images restated (importing ertm.pipeline needs matplotlib)."""
    rng = np.random.default_rng(21)
    imgs = [rng.normal(scale=s, size=(19, 23)).astype(np.float32) for s in (1.0, 3.0, 0.2)]
    stacked = np.zeros(imgs[0].shape, dtype=np.float64)
    for im in imgs:
        d = np.asarray(im, dtype=np.float64)
        sc = float(np.max(np.abs(d)))
        stacked += d / sc if sc > 0 else d
    stacked /= len(imgs)
    return {"images": np.stack(imgs), "stacked": stacked.astype(np.float32)}


def preprocess_case() -> dict[str, np.ndarray]:
    """preprocess.py:36-224: rotation, sinc resampling (up and down), direct-wave
    mute, end taper and the combined prepare_shot, on a seeded 3-component shot."""
    from ertm import preprocess as pre
    from ertm.types import ShotRecord
    rng = np.random.default_rng(31)
    nt, nrec, dt = 240, 19, 4e-4
    rec = receivers_line(0.0, 540.0, nrec, 8.0)
    src = SourceSpec(x=260.0, z=12.0, f0=30.0, delay=0.03)
    t = np.arange(nt) * dt
    comps = {n: (rng.normal(size=(nt, nrec)) * s).astype(np.float32) for n, s in (("p", 1.0), ("vx", 0.3),
                                                                                  ("vz", 0.5))}
    shot = ShotRecord(data=comps["p"], dt=dt, t=t, receivers=rec, source=src, components=dict(comps))
    model = layered_model(60, 40, 10.0, 5)
    out = {"nt": np.array(nt), "dt": np.array(dt), "rx": rec.x, "rz": rec.z,
           "src": np.array([src.x, src.z, src.f0, src.delay, src.amplitude])}
    out.update({f"in_{n}": v for n, v in comps.items()})
    out.update(model_arrays("m_", model))
    rot = pre.rotate_components(comps, 30.0)
    out.update({f"rot_{n}": np.asarray(v) for n, v in rot.items()})
    for tag, dt_out in (("up", 3e-4), ("down", 5.5e-4)):
        r = pre.resample_shot(shot, dt_out)
        out.update({f"res_{tag}_{n}": np.asarray(v) for n, v in r.components.items()})
        out[f"res_{tag}_data"] = np.asarray(r.data)
    m = pre.mute_direct_wave(shot, 2100.0)
    out.update({f"mute_{n}": np.asarray(v) for n, v in m.components.items()})
    out["mute_data"] = np.asarray(m.data)
    tp = pre.taper_record_ends(shot, 0.05)
    out.update({f"taper_{n}": np.asarray(v) for n, v in tp.components.items()})
    out["taper_data"] = np.asarray(tp.data)
    ps = pre.prepare_shot(shot, model=model, record_dt=3.5e-4, rotation_deg=25.0, mute=True, taper_fraction=0.05)
    out.update({f"prep_{n}": np.asarray(v) for n, v in ps.components.items()})
    out["prep_data"] = np.asarray(ps.data)
    out["prep_dt"] = np.array(ps.dt)
    return out


def qcomp_case() -> dict[str, np.ndarray]:
    """qcomp.py:98-213: receiver-side compensation (the migrate preprocess hook)
    and constant-Q attenuation through the short-time overlap-add filter."""
    from ertm.qcomp import QCompensator, attenuate_record
    rng = np.random.default_rng(41)
    data = rng.normal(size=(300, 7)).astype(np.float32)
    comp = QCompensator(config=QConfig(enabled=True, model="filter", alpha_c=0.8, gain_cap=30.0, f_ref=30.0),
                        q_value=60.0)
    return {"data": data, "dt": np.array(1e-3), "compensated": comp(data.astype(np.float64), 1e-3),
            "attenuated": attenuate_record(data, 1e-3, 50.0, f_ref=30.0, nperseg=64),
            "trace": attenuate_record(data[:, 0], 1e-3, 80.0, nperseg=96)}


def store_case() -> dict[str, np.ndarray]:
    """data.py:73-297: the reference's NumpyDataStore writes one model, one
    three-component shot and one image; the three .npz files are committed
    under tests/golden/store/ as written, and this case holds what went in."""
    import shutil
    import tempfile

    from ertm.data import NumpyDataStore
    from ertm.types import ImageResult, ShotRecord
    model = layered_model(19, 13, 10.0, seed=5)
    model.name, model.meta = "store-model", {"builder": "layered", "layers": 3}
    rng = np.random.default_rng(9)
    nt, nrec = 40, 6
    comps = {n: rng.normal(size=(nt, nrec)).astype(np.float32) for n in ("p", "vx", "vz")}
    shot = ShotRecord(data=comps["p"], dt=5e-4, t=np.arange(nt) * 5e-4,
                      receivers=ReceiverSpec(x=np.linspace(10.0, 160.0, nrec), z=np.full(nrec, 20.0), component="p"),
                      source=SourceSpec(x=90.0, z=20.0, f0=25.0, amplitude=2.0, delay=0.01, mechanism="shear"),
                      meta={"synthetic": True, "engine": "elastic"}, components=comps)
    image = ImageResult(image=rng.normal(size=model.grid.shape).astype(np.float32), grid=model.grid, mode="ps",
                        meta={"condition": "normalized", "n_shots": 3})
    out = HERE / "store"
    out.mkdir(exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        store = NumpyDataStore(tmp)
        for written in (store.save_model(model, "model"), store.save_shot(shot, "shot"),
                        store.save_image(image, "image")):
            shutil.copyfile(written, out / written.name)
    return {"vp": model.vp, "vs": model.vs, "rho": model.rho, "qp": model.qp, "qs": model.qs,
            "grid": np.array([19, 13, 10.0, 10.0, 0.0, 0.0]), "data": shot.data, "t": shot.t,
            "rx": shot.receivers.x, "rz": shot.receivers.z, "comp_p": comps["p"], "comp_vx": comps["vx"],
            "comp_vz": comps["vz"], "image": image.image}


def main() -> None:
    cases = {
        "store": store_case,
        "qcomp": qcomp_case,
        "preprocess": preprocess_case,
        "numerics": numerics_case,
        "gsls": gsls_case,
        "acoustic_cpml": lambda: propagate_case("acoustic", "cpml", nt=90, inject_every=7),
        "acoustic_free": lambda: propagate_case("acoustic", "free", nt=90),
        "acoustic_none": lambda: propagate_case("acoustic", "none", nt=40),
        "elastic_free_explosive": lambda: propagate_case("elastic", "free", nt=80, inject_every=9),
        "elastic_cpml_shear": lambda: propagate_case("elastic", "cpml", nt=60, mechanism="shear"),
        "elastic_free_forcez": lambda: propagate_case("elastic", "free", nt=60, mechanism="force_z"),
        "visco_cpml": lambda: propagate_case(
            "viscoacoustic", "cpml", nt=80, q=QOptions(enabled=True, f_ref=25.0), inject_every=11),
        "visco_comp_free": lambda: propagate_case(
            "viscoacoustic", "free", nt=90,
            q=QOptions(enabled=True, f_ref=25.0, compensation=True, amplitude_cap=1.5,
                       lowpass_interval=20, f_max=60.0, gain_budget_db=40.0)),
        "mig_acoustic_zerolag": lambda: migrate_case("acoustic", "zero_lag", boundary="cpml"),
        "mig_acoustic_norm_rn": lambda: migrate_case(
            "acoustic", "normalized", boundary="free", receiver_normalization=True),
        "mig_acoustic_excitation": lambda: migrate_case(
            "acoustic", "excitation", boundary="free", receiver_normalization=True),
        "mig_elastic_pp_divcurl": lambda: migrate_case(
            "elastic", "normalized", boundary="free", mode="pp", nt=220,
            components=("p", "vx", "vz", "sxz")),
        "mig_elastic_ps_stress": lambda: migrate_case(
            "elastic", "zero_lag", boundary="cpml", mode="ps", separation="stress", nt=220,
            components=("vx", "vz")),
        "mig_visco_comp": lambda: migrate_case(
            "viscoacoustic", "normalized", boundary="free", nt=240,
            q=QConfig(enabled=True, model="gsls", alpha_c=1.0, f_ref=25.0, f_max=60.0,
                      gain_budget_db=40.0, amplitude_cap=50.0, lowpass_interval=20)),
        "stack": stack_case,
    }
    only = set(sys.argv[2:])
    for name, fn in cases.items():
        if only and name not in only:
            continue
        arrays = fn()
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        size = (HERE / f"{name}.npz").stat().st_size
        print(f"{name}: {len(arrays)} arrays, {size / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
