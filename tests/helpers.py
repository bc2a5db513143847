"""Shared test helpers: golden-fixture loading and duck-typed inputs."""

from __future__ import annotations

import json
from pathlib import Path
from types import SimpleNamespace

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        out = {k: z[k] for k in z.files}
    if "meta" in out:
        out["meta"] = json.loads(str(out["meta"]))
    return out


def model_from(fx: dict, prefix: str = "m_") -> SimpleNamespace:
    nx, nz, dx, dz, x0, z0 = fx[f"{prefix}grid"]
    grid = SimpleNamespace(nx=int(nx), nz=int(nz), dx=float(dx), dz=float(dz), x0=float(x0),
                           z0=float(z0), shape=(int(nz), int(nx)))
    return SimpleNamespace(grid=grid, vp=fx[f"{prefix}vp"], vs=fx[f"{prefix}vs"], rho=fx[f"{prefix}rho"],
                           qp=fx[f"{prefix}qp"], qs=fx[f"{prefix}qs"], shape=grid.shape)


def source_from(fx: dict, mechanism: str = "explosive") -> SimpleNamespace:
    x, z, f0, delay, amp = fx["src"]
    return SimpleNamespace(x=float(x), z=float(z), f0=float(f0), delay=float(delay),
                           amplitude=float(amp), kind="ricker", mechanism=mechanism)


def receivers_from(fx: dict) -> SimpleNamespace:
    return SimpleNamespace(x=np.asarray(fx["rx"], dtype=float), z=np.asarray(fx["rz"], dtype=float),
                           component="p")


def q_from(meta_q: dict | None) -> SimpleNamespace | None:
    if meta_q is None:
        return None
    return SimpleNamespace(**meta_q)


def imaging_from(meta: dict) -> SimpleNamespace:
    """ImagingConfig defaults (config.py:310-351) overridden by the case."""
    return SimpleNamespace(mode=meta["mode"], condition=meta["condition"], separation=meta["separation"],
                           illumination=True, receiver_normalization=meta["receiver_normalization"],
                           laplacian=True, lowpass_fraction=meta["lowpass"],
                           checkpoint_mb=meta["checkpoint_mb"], eps=1e-10, start_periods=1.5)


def solver_from(meta: dict) -> SimpleNamespace:
    return SimpleNamespace(nt=meta["nt"], dt=meta["dt"], order=8, boundary=meta["boundary"],
                           dtype="float32", engine=meta["engine"], npml=12)


def q_options_for_migrate(meta_q: dict | None) -> SimpleNamespace | None:
    """RTMImager.q_options (imaging.py:187-202): QConfig → QOptions fields."""
    if meta_q is None:
        return None
    return SimpleNamespace(enabled=True, f_ref=meta_q["f_ref"], n_mechanisms=meta_q["n_mechanisms"],
                           band_ratio=meta_q["band_ratio"], compensation=bool(meta_q["enabled"]),
                           alpha_c=meta_q["alpha_c"], amplitude_cap=meta_q["amplitude_cap"],
                           lowpass_interval=meta_q["lowpass_interval"], f_max=meta_q["f_max"],
                           gain_budget_db=meta_q["gain_budget_db"])


PROPAGATION_CASES = [
    "acoustic_cpml", "acoustic_free", "acoustic_none",
    "elastic_free_explosive", "elastic_cpml_shear", "elastic_free_forcez",
    "visco_cpml", "visco_comp_free",
]
MIGRATE_CASES = [
    "mig_acoustic_zerolag", "mig_acoustic_norm_rn", "mig_acoustic_excitation",
    "mig_elastic_pp_divcurl", "mig_elastic_ps_stress", "mig_visco_comp",
]


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))
