"""Seeded synthetic earth models and acquisitions for benchmarking.

There is no public dataset for this path; these builders produce models with
the shapes, sizes and value ranges of the benchmark configurations:

* ``elastic_borehole_4c`` — 401×601 at 5 m, 6–10 layers with vp 2500–4500
  m/s, vs = vp/1.73, Gardner density, six circular cavities (r 10–30 m,
  vp 1500 m/s) and one 60° fault with 50 m throw; 8 surface shots; 100 4C
  receivers in a well at x = 1000 m, z = 500…2480 m.  Two adjustments keep
  the reference's own checks passing: dt is the CFL limit at safety 0.5
  (≈0.305 ms, 1.5 s → 4912 steps) instead of 0.5 ms, and cavities get
  vs = 1e-3·vp instead of 0 (the model contract needs vs > 0).
* ``acoustic_layered`` — 301×201 at 10 m, interfaces at 700/1300 m with vp
  2000/2500/3000 m/s, 3 shots, 150 receivers at 2 m depth, dt 1 ms, 1500 steps.
* ``visco_layered`` — L=3 GSLS, 2001×801 at 5 m, layered vp 1800–4000 m/s,
  Q 30–200 log-uniform per layer, 30 Hz source, 400 receivers per shot.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .numerics import cfl_dt
from .types import ElasticModel, GridSpec, ReceiverSpec, SourceSpec


def gardner(vp: np.ndarray) -> np.ndarray:
    return (310.0 * np.asarray(vp, dtype=np.float64) ** 0.25).astype(np.float32)


@dataclass
class Workload:
    name: str
    engine: str
    model: ElasticModel
    sources: list[SourceSpec]
    receivers: ReceiverSpec
    dt: float
    nt: int
    boundary: str
    npml: int
    condition: str
    separation: str = "divcurl"
    modes: tuple[str, ...] = ("pp",)
    components: tuple[str, ...] = ("p",)
    checkpoint_mb: float = 256.0
    q: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.model.grid.nx * self.model.grid.nz


def elastic_borehole_4c(seed: int = 0, n_shots: int = 8, nt: int | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    nx, nz, h = 401, 601, 5.0
    grid = GridSpec(nx=nx, nz=nz, dx=h, dz=h)
    x = np.arange(nx) * h
    z = np.arange(nz) * h
    xx, zz = np.meshgrid(x, z)
    n_layers = int(rng.integers(6, 11))
    tops = np.sort(rng.uniform(150.0, (nz - 20) * h, n_layers - 1))
    vps = np.sort(rng.uniform(2500.0, 4500.0, n_layers))
    vps[0], vps[-1] = 2500.0, 4500.0
    # 60° fault through (x_f, z_f); the hanging wall is thrown down by 50 m
    x_f, z_f = float(rng.uniform(700.0, 1300.0)), float(rng.uniform(800.0, 2200.0))
    hanging = xx > x_f + (zz - z_f) / np.tan(np.deg2rad(60.0))
    depth = np.where(hanging, zz - 50.0, zz)
    layer = np.searchsorted(tops, depth)
    vp = vps[layer]
    vs = vp / 1.73
    for _ in range(6):
        cx, cz, r = rng.uniform(200.0, 1800.0), rng.uniform(400.0, 2800.0), rng.uniform(10.0, 30.0)
        hole = (xx - cx) ** 2 + (zz - cz) ** 2 <= r * r
        vp = np.where(hole, 1500.0, vp)
        vs = np.where(hole, 1.5, vs)          # 1e-3·vp: the model contract needs vs > 0
    vp = vp.astype(np.float32)
    vs = vs.astype(np.float32)
    model = ElasticModel(grid=grid, vp=vp, vs=vs, rho=gardner(vp), qp=np.full(grid.shape, 100.0, np.float32),
                         qs=np.full(grid.shape, 50.0, np.float32), name="elastic-borehole-4c")
    dt = cfl_dt(4500.0, h, h, 8, 0.5)
    steps = int(round(1.5 / dt)) if nt is None else int(nt)
    xs = np.sort(rng.uniform(100.0, 1900.0, n_shots))
    sources = [SourceSpec(x=float(v), z=20.0, f0=25.0, delay=0.08) for v in xs]
    zr = np.arange(500.0, 2481.0, 20.0)
    receivers = ReceiverSpec(x=np.full_like(zr, 1000.0), z=zr, component="vz")
    return Workload("elastic borehole 4C PP/PS (401x601, 8 shots)", "elastic", model, sources, receivers, dt, steps,
                    "free", 40, "normalized", separation="divcurl", modes=("pp", "ps"),
                    components=("p", "vx", "vz", "sxz"), checkpoint_mb=256.0)


def acoustic_layered(seed: int = 0, n_shots: int = 3, nt: int | None = None) -> Workload:
    nx, nz, h = 301, 201, 10.0
    grid = GridSpec(nx=nx, nz=nz, dx=h, dz=h)
    z = np.arange(nz)[:, None] * h
    vp = np.where(z < 700.0, 2000.0, np.where(z < 1300.0, 2500.0, 3000.0)).repeat(nx, 1).astype(np.float32)
    model = ElasticModel(grid=grid, vp=vp, vs=(vp / 1.73).astype(np.float32), rho=gardner(vp),
                         qp=np.full(grid.shape, 100.0, np.float32), qs=np.full(grid.shape, 50.0, np.float32),
                         name="acoustic-3-layer")
    xs = [750.0, 1500.0, 2250.0][:n_shots] if n_shots <= 3 else list(np.linspace(300.0, 2700.0, n_shots))
    sources = [SourceSpec(x=float(v), z=20.0, f0=15.0, delay=0.08) for v in xs]
    xr = np.arange(0.0, 2981.0, 20.0)
    receivers = ReceiverSpec(x=xr, z=np.full_like(xr, 2.0), component="p")
    return Workload("acoustic 3-layer zero-lag (301x201, 3 shots)", "acoustic", model, sources, receivers, 1e-3,
                    1500 if nt is None else int(nt), "cpml", 30, "zero_lag", checkpoint_mb=64.0)


def visco_layered(seed: int = 0, n_shots: int = 64, nt: int | None = None, nx: int = 2001, nz: int = 801,
                  n_receivers: int = 400) -> Workload:
    rng = np.random.default_rng(seed)
    h = 5.0
    grid = GridSpec(nx=nx, nz=nz, dx=h, dz=h)
    n_layers = int(rng.integers(5, 9))
    tops = np.sort(rng.uniform(100.0, (nz - 10) * h, n_layers - 1))
    vps = np.sort(rng.uniform(1800.0, 4000.0, n_layers))
    vps[0], vps[-1] = 1800.0, 4000.0
    qs = np.exp(rng.uniform(np.log(30.0), np.log(200.0), n_layers))
    layer = np.searchsorted(tops, np.arange(nz) * h)
    vp = vps[layer][:, None].repeat(nx, 1).astype(np.float32)
    qp = np.round(qs[layer])[:, None].repeat(nx, 1).astype(np.float32)
    model = ElasticModel(grid=grid, vp=vp, vs=(vp / 1.8).astype(np.float32), rho=gardner(vp), qp=qp,
                         qs=(qp * 0.5).astype(np.float32), name="visco-gsls-layered")
    dt = 0.34e-3
    steps = int(round(1.6 / dt)) if nt is None else int(nt)
    xs = 150.0 + 150.0 * np.arange(n_shots)
    sources = [SourceSpec(x=float(v), z=20.0, f0=30.0, delay=0.06) for v in xs]
    xr = np.linspace(0.0, (nx - 1) * h, n_receivers)
    receivers = ReceiverSpec(x=xr, z=np.full_like(xr, 2.0), component="p")
    return Workload("viscoacoustic GSLS L=3 with Q compensation", "viscoacoustic", model, sources, receivers, dt, steps,
                    "cpml", 20, "normalized", q=dict(enabled=True, model="gsls", alpha_c=1.0, f_ref=30.0,
                                                       gain_budget_db=40.0, f_max=60.0, amplitude_cap=50.0,
                                                       lowpass_interval=20, n_mechanisms=3))


WORKLOADS = {"elastic4c": elastic_borehole_4c, "acoustic": acoustic_layered, "visco": visco_layered}


UNEVEN_GRIDS = ((501, 301), (1001, 501), (1601, 801), (2401, 1201))


def uneven_batch(seed: int = 0, n_shots: int = 256, *, h: float = 10.0) -> list[Workload]:
    """Uneven batch: one single-shot workload per shot.

    Engine uniform over acoustic / elastic; the model one of four seeded
    random-layer models with an anomaly (501×301, 1001×501, 1601×801,
    2401×1201 at 10 m); dt at the CFL limit (safety 0.5); nt uniform in
    1500–6000; 10–30 Hz Ricker; normalized condition (the batch is run with
    Kahan-compensated float32 accumulation)."""
    rng = np.random.default_rng(seed)
    models = []
    for k, (nx, nz) in enumerate(UNEVEN_GRIDS):
        grid = GridSpec(nx=nx, nz=nz, dx=h, dz=h)
        n_layers = int(rng.integers(4, 9))
        tops = np.sort(rng.uniform(0.05, 0.95, n_layers - 1)) * nz * h
        vps = np.sort(rng.uniform(1800.0, 4200.0, n_layers))
        layer = np.searchsorted(tops, np.arange(nz) * h)
        vp = vps[layer][:, None].repeat(nx, 1)
        # anomaly: an elliptic body 15 % faster or slower than its layer
        cx, cz = rng.uniform(0.3, 0.7) * nx * h, rng.uniform(0.4, 0.8) * nz * h
        ax, az = rng.uniform(0.05, 0.15) * nx * h, rng.uniform(0.03, 0.08) * nz * h
        xx, zz = np.meshgrid(np.arange(nx) * h, np.arange(nz) * h)
        body = ((xx - cx) / ax) ** 2 + ((zz - cz) / az) ** 2 <= 1.0
        vp = np.where(body, vp * (1.15 if rng.uniform() < 0.5 else 0.85), vp).astype(np.float32)
        models.append(ElasticModel(grid=grid, vp=vp, vs=(vp / 1.8).astype(np.float32), rho=gardner(vp),
                                   qp=np.full(grid.shape, 100.0, np.float32), qs=np.full(grid.shape, 50.0, np.float32),
                                   name=f"uneven-{nx}x{nz}"))
    out = []
    for i in range(n_shots):
        engine = ("acoustic", "elastic")[int(rng.integers(0, 2))]
        m = models[int(rng.integers(0, len(models)))]
        g = m.grid
        nt = int(rng.integers(1500, 6001))
        f0 = float(rng.uniform(10.0, 30.0))
        dt = cfl_dt(float(m.vp.max()), g.dx, g.dz, 8, 0.5)
        src = SourceSpec(x=float(rng.uniform(0.05, 0.95) * (g.nx - 1) * h), z=2.0 * h, f0=f0, delay=1.2 / f0)
        xr = np.arange(0, g.nx, 4) * h
        rec = ReceiverSpec(x=xr, z=np.full_like(xr, 2.0 * h), component="p")
        boundary = "free" if engine == "elastic" else "cpml"
        comps = ("vz", "p") if engine == "elastic" else ("p",)
        modes = ("pp", "ps") if engine == "elastic" else ("pp",)
        out.append(Workload(f"uneven shot {i}: {engine} {g.nx}x{g.nz} nt={nt}", engine, m, [src], rec, dt, nt, boundary,
                            20, "normalized", separation="divcurl", modes=modes, components=comps,
                            checkpoint_mb=256.0))
    return out

def imager_for(wl: Workload):
    """The RTMImager (and its SolverConfig) a workload is migrated with."""
    from .config import ImagingConfig, QConfig, SolverConfig
    from .imaging import RTMImager
    solver = SolverConfig(nt=wl.nt, dt=wl.dt, order=8, boundary=wl.boundary, dtype="float32", engine=wl.engine,
                          npml=wl.npml)
    imaging = ImagingConfig(mode=wl.modes[0], condition=wl.condition, separation=wl.separation,
                            checkpoint_mb=wl.checkpoint_mb)
    q = QConfig(**wl.q) if wl.q else None
    return RTMImager(imaging, solver, q), solver


def synthesize(wl: Workload, solver, sources):
    """Shot records of ``sources`` from the GPU forward model (with the
    workload's Q settings for the viscoacoustic engine)."""
    from .config import QConfig
    from .solver import FiniteDifferenceSolver
    fd = FiniteDifferenceSolver(solver, QConfig(**wl.q) if wl.q else None)
    return [fd.forward(wl.model, s, wl.receivers, components=wl.components) for s in sources]


def serving_jobs(seed: int = 0, n_jobs: int = 32, *, max_scale: tuple[float, float] = (16.0, 8.0),
                 nt_range: tuple[int, int] = (1000, 8000), max_shots: int = 16):
    """A stream of migration jobs of mixed engine, grid and length.

    Engine uniform over acoustic / elastic / viscoacoustic; grid 256·u × 256·v
    with u, v log-uniform in [1, max_scale] (the full range is 256×256 to
    4096×2048); spacing 5–10 m; random layered vp 1500–4000 m/s with Gardner
    density and layered Q 30–200; dt at the CFL limit (safety 0.5); length
    uniform in nt_range; 1..max_shots surface shots with 10–30 Hz Ricker
    wavelets; receivers every 4 cells at 2 cells depth.  Records are seeded
    noise (the work of a shot does not depend on the record's values).
    Returns ``ServeJob`` objects."""
    from .config import ImagingConfig, QConfig, SolverConfig
    from .imaging import RTMImager
    from .serving import ServeJob
    from .types import ShotRecord
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_jobs):
        engine = ("acoustic", "elastic", "viscoacoustic")[int(rng.integers(0, 3))]
        nx = int(round(256 * np.exp(rng.uniform(0.0, np.log(max_scale[0])))))
        nz = int(round(256 * np.exp(rng.uniform(0.0, np.log(max_scale[1])))))
        h = float(rng.integers(5, 11))
        grid = GridSpec(nx=nx, nz=nz, dx=h, dz=h)
        n_layers = int(rng.integers(3, 7))
        tops = np.sort(rng.uniform(0.1, 0.95, n_layers - 1)) * nz * h
        vps = np.sort(rng.uniform(1500.0, 4000.0, n_layers))
        qs = np.round(np.exp(rng.uniform(np.log(30.0), np.log(200.0), n_layers)))
        layer = np.searchsorted(tops, np.arange(nz) * h)
        vp = vps[layer][:, None].repeat(nx, 1).astype(np.float32)
        qp = qs[layer][:, None].repeat(nx, 1).astype(np.float32)
        model = ElasticModel(grid=grid, vp=vp, vs=(vp / 1.8).astype(np.float32), rho=gardner(vp), qp=qp,
                             qs=(qp * 0.5).astype(np.float32), name=f"serving-{j}")
        dt = cfl_dt(float(vps.max()), h, h, 8, 0.5)
        nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
        f0 = float(rng.uniform(10.0, 30.0))
        boundary = "free" if engine == "elastic" else "cpml"
        solver = SolverConfig(nt=nt, dt=dt, order=8, boundary=boundary, engine=engine)
        q = QConfig(enabled=True, model="gsls", alpha_c=1.0, f_ref=f0, gain_budget_db=40.0, f_max=2.0 * f0,
                    amplitude_cap=50.0, lowpass_interval=20, n_mechanisms=3) if engine == "viscoacoustic" else None
        imaging = ImagingConfig(mode="pp", condition="normalized", separation="divcurl", checkpoint_mb=256.0)
        imager = RTMImager(imaging, solver, q)
        xr = np.arange(0, nx, 4) * h
        receivers = ReceiverSpec(x=xr, z=np.full_like(xr, 2.0 * h), component="p")
        comps = ("vz", "p") if engine == "elastic" else ("p",)
        shots = []
        for k in range(int(rng.integers(1, max_shots + 1))):
            src = SourceSpec(x=float(rng.uniform(0.1, 0.9) * (nx - 1) * h), z=2.0 * h, f0=f0, delay=1.2 / f0)
            data = {c: (rng.standard_normal((nt, len(xr))) * 1e-6).astype(np.float32) for c in comps}
            shots.append(ShotRecord(data=data[comps[0]], dt=dt, t=np.arange(nt) * dt, receivers=receivers,
                                    source=src, components=data))
        modes = ("pp", "ps") if engine == "elastic" else ("pp",)
        jobs.append(ServeJob(shots=shots, model=model, imager=imager, modes=modes,
                             name=f"{engine} {nx}x{nz} nt={nt} shots={len(shots)}"))
    return jobs


def serving_workload(index: int, seed: int = 1, *, max_scale: tuple[float, float] = (16.0, 8.0),
                     nt_range: tuple[int, int] = (1000, 8000), max_shots: int = 16) -> Workload:
    """Job ``index`` of the serving stream ``serving_jobs(seed, …)`` as a
    workload (its model, sources, receivers, time axis and imaging settings;
    records are then synthesised rather than the stream's noise)."""
    job = serving_jobs(seed=seed, n_jobs=index + 1, max_scale=max_scale, nt_range=nt_range,
                       max_shots=max_shots)[index]
    solver = job.imager.solver_config
    imaging = job.imager.config
    q = job.imager.q_config
    qd = {}
    if solver.engine == "viscoacoustic":
        qd = dict(enabled=True, model="gsls", alpha_c=q.alpha_c, f_ref=q.f_ref, gain_budget_db=q.gain_budget_db,
                  f_max=q.f_max, amplitude_cap=q.amplitude_cap, lowpass_interval=q.lowpass_interval,
                  n_mechanisms=q.n_mechanisms)
    shot0 = job.shots[0]
    comps = tuple(shot0.components) if shot0.components else ("p",)
    return Workload(f"serving job {index}: {job.name}", solver.engine, job.model, [s.source for s in job.shots],
                    shot0.receivers, float(solver.dt), int(solver.nt), solver.boundary, int(solver.npml),
                    imaging.condition, separation=imaging.separation, modes=tuple(job.modes), components=comps,
                    checkpoint_mb=float(imaging.checkpoint_mb), q=qd)
