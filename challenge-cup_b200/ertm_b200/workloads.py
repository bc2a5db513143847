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
