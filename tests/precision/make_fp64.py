"""FP64 oracle images for the precision study (imaging in float32 wavefields
on the device against float64 wavefields on the host).

Runs on the CPU, with the oracle.  For a few seeded shots of each benchmark
configuration it

* synthesises the shot record with the oracle's float32 forward model (the
  device forward model reproduces it bit for bit for the acoustic and elastic
  engines, and to float32 rounding for the viscoacoustic one);
* migrates it with the oracle in float64 wavefields (the reference's float64
  mode: CPML coefficients and ψ memories stay float32, propagation.py
  ``dtype="float64"``), imaging and post-processing as the path does;
* stores the images every ``step``-th pixel in both axes as float32.

Output: tests/precision/<config>.npz.  The device side of the comparison is
tests/test_gpu_precision.py.

    python tests/precision/make_fp64.py [config ...]     # acoustic elastic4c visco uneven
    python tests/precision/make_fp64.py --float32 visco  # the same in float32 wavefields (<config>_f32.npz)
"""

from __future__ import annotations

import json
import multiprocessing as mp
import sys
import time
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

# config: (shot indices, decimation step, stack the shots, workload overrides).
# The viscoacoustic study uses a 2 GiB checkpoint budget on both sides: at the
# default 256 MB the oracle's float64 replay block (2353 steps of 1.6 M-cell
# image fields) needs 30 GB of host memory per shot.
CASES = {
    "acoustic": ([0, 1, 2], 2, True, {}),
    "elastic4c": ([0, 5], 4, False, {}),
    "visco": ([10, 40], 8, False, {"checkpoint_mb": 2048.0}),
    "uneven": ([1, 4], 4, False, {}),
    # a compensated viscoacoustic job of the serving stream (job 13 of the
    # full-scale stream: 396x1378, nt 1586), its first shot
    "serving": ([0], 4, False, {}),
}


def _paths() -> None:
    for p in (str(ROOT), str(ROOT / "challenge-cup_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)


def case_workloads(config: str):
    """The single-shot workloads of one configuration's study (also used by
    the device test, so both sides see the same seeded inputs)."""
    _paths()
    from ertm_b200 import workloads
    shots, _, _, over = CASES[config]
    if config == "uneven":
        batch = workloads.uneven_batch(0, 8)
        return [workloads.Workload(**{**batch[i].__dict__, **over}) for i in shots]
    if config == "serving":
        wl = workloads.serving_workload(13)
        return [workloads.Workload(**{**wl.__dict__, "sources": [wl.sources[i]], **over}) for i in shots]
    wl = workloads.WORKLOADS[config](seed=0)
    return [workloads.Workload(**{**wl.__dict__, "sources": [wl.sources[i]], **over}) for i in shots]


def _oracle_q(qcfg, compensation: bool):
    return SimpleNamespace(enabled=True, f_ref=float(qcfg.f_ref), n_mechanisms=int(qcfg.n_mechanisms),
                           band_ratio=float(qcfg.band_ratio), compensation=bool(compensation),
                           alpha_c=float(qcfg.alpha_c), amplitude_cap=float(qcfg.amplitude_cap),
                           lowpass_interval=int(qcfg.lowpass_interval),
                           f_max=None if qcfg.f_max is None else float(qcfg.f_max),
                           gain_budget_db=float(qcfg.gain_budget_db))


def run_shot(args) -> dict:
    config, k, dtype = args
    _paths()
    import oracle as orc
    from ertm_b200 import workloads
    wl = case_workloads(config)[k]
    imager, solver = workloads.imager_for(wl)
    t0 = time.perf_counter()
    spec = orc.Spec(dt=wl.dt, nt=wl.nt, order=8, npml=wl.npml, dtype="float32", boundary=wl.boundary)
    q_fwd = _oracle_q(imager.q_config, False) if wl.engine == "viscoacoustic" else None
    record = orc.run_forward(wl.model, wl.sources[0], wl.receivers, spec, engine=wl.engine,
                             components=list(wl.components), q=q_fwd)
    t1 = time.perf_counter()
    sv = SimpleNamespace(dt=wl.dt, nt=wl.nt, order=8, boundary=wl.boundary, dtype=dtype, engine=wl.engine,
                         npml=wl.npml)
    q = _oracle_q(imager.q_config, bool(imager.q_config.enabled)) if wl.engine == "viscoacoustic" else None
    images = {}
    for m in wl.modes:
        im = SimpleNamespace(**{**imager.config.__dict__, "mode": m})
        images[m] = np.asarray(orc.migrate(record, wl.dt, wl.sources[0], wl.receivers, wl.model, sv, im, q),
                               dtype=np.float64)
    return {"config": config, "k": k, "images": images, "forward_s": t1 - t0,
            "migrate_s": time.perf_counter() - t1, "dtype": dtype}


def save(config: str, results: list[dict], suffix: str = "") -> None:
    import oracle as orc
    shots, step, stack, over = CASES[config]
    rs = sorted(results, key=lambda r: r["k"])
    modes = sorted({m for r in rs for m in r["images"]})
    meta = {"shots": shots, "step": step, "stacked": stack, "modes": modes, "overrides": over,
            "forward_s": [r["forward_s"] for r in rs], "migrate_s": [r["migrate_s"] for r in rs],
            "wavefields": rs[0]["dtype"]}
    out = {}
    for m in modes:
        if stack:
            imgs = [r["images"][m] for r in rs]
            out[m] = orc.stack_images(imgs, normalize=True)[::step, ::step].astype(np.float32)
        else:
            for r in rs:
                if m in r["images"]:
                    out[f"{m}_{r['k']}"] = r["images"][m][::step, ::step].astype(np.float32)
    np.savez_compressed(HERE / f"{config}{suffix}.npz", meta=json.dumps(meta), **out)
    print(config, json.dumps(meta), flush=True)


def main(configs, dtype: str = "float64") -> None:
    _paths()
    tasks = [(c, k, dtype) for c in configs for k in range(len(CASES[c][0]))]
    ctx = mp.get_context("spawn")
    done: dict[str, list] = {c: [] for c in configs}
    suffix = "" if dtype == "float64" else "_f32"
    with ctx.Pool(min(len(tasks), mp.cpu_count())) as pool:
        for r in pool.imap_unordered(run_shot, tasks):
            done[r["config"]].append(r)
            if len(done[r["config"]]) == len(CASES[r["config"]][0]):
                save(r["config"], done[r["config"]], suffix)


if __name__ == "__main__":
    # --float32: the oracle's migrate in float32 wavefields (the reference's own
    # precision), written as <config>_f32.npz beside the float64 images
    args = [a for a in sys.argv[1:] if a != "--float32"]
    main(args or list(CASES), "float32" if "--float32" in sys.argv[1:] else "float64")
