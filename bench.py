#!/usr/bin/env python
"""Benchmark of the B200 RTM hot path.

Default workload (one GPU): the viscoacoustic GSLS configuration with Q
compensation - 2001×801 grid at 5 m, L = 3 relaxation mechanisms, layered
vp 1800-4000 m/s and Q 30-200, 64 surface shots 150 m apart with 400
receivers each, 4706 steps (1.6 s at dt 0.34 ms), 30 Hz Ricker, normalized
condition, compensation with α_c = 1, 40 dB gain budget and f_max 60 Hz.
The job's 64 shots are migrated four per benchmark step (the step's shots
advance together in lockstep ticks) and each step's images are stacked; the
steps cycle through the job's shots.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
    python bench.py --gpus N ...      (no torchrun: the benchmark starts N
        ranks itself, one per GPU; weak scaling - every rank migrates its own
        shots per step, one NCCL all-reduce of the float64 stack per step)

One JSON line is printed by rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT), str(ROOT / "challenge-cup_b200")]

import numpy as np  # noqa: E402

METRIC = "shots/s & Gcell-updates/s batched vs plain on 1 B200; p99 latency @ 1e-4 err"
FALLBACK_HBM_GBS = 6650.0
SHOTS_PER_STEP = {"visco": 4, "elastic4c": 8, "acoustic": 3}


def parse_args(argv=None) -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", default="visco", choices=sorted(SHOTS_PER_STEP))
    ap.add_argument("--nt", type=int, default=None, help="override the number of time steps (profiling runs)")
    ap.add_argument("--shots", type=int, default=None, help="override the shots per rank and step")
    ap.add_argument("--plain-steps", type=int, default=3, help="timed steps of the plain one-shot arm")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=48)
    ap.add_argument("--serve-jobs", type=int, default=24, help="jobs in the serving run (0: no serving run)")
    ap.add_argument("--serve-scale", choices=("short", "full"), default="short",
                    help="short: grids up to 1024x512, nt 500-2000, 1-4 shots (seconds); full: the serving "
                         "configuration (grids up to 4096x2048, nt 1000-8000, 1-16 shots, minutes)")
    ap.add_argument("--serving-only", action="store_true",
                    help="run only the serving stream (--serve-jobs, --serve-scale) and print its JSON")
    ap.add_argument("--uneven-shots", type=int, default=24,
                    help="shots of the uneven batch (256-shot configuration) timed batched vs plain (0: skip)")
    ap.add_argument("--no-adjacent", action="store_true",
                    help="skip timing the steps either side of the path (preprocessing, Q filter, SEG-Y, stack)")
    return ap.parse_args(argv)


def launch_ranks(args) -> int:
    """`--gpus N` without a launcher: start N ranks (one per GPU) through
    torch.distributed.run on 127.0.0.1 and return rank 0's exit status."""
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve()), *sys.argv[1:]]
    try:   # a last bound well above the process group's own timeout
        return subprocess.call(cmd, timeout=3600)
    except subprocess.TimeoutExpired:
        print(json.dumps({"error": "ranks did not finish within 3600 s"}), flush=True)
        return 1


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self, join: bool = True) -> None:
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1 and join:
            import datetime

            import torch
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            # short enough that ranks left waiting on a failed peer end with an error
            # (the longest gap between collectives is the per-rank set-up, well under it)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self) -> None:
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum_(self, t) -> None:
        if self.pg:
            self.pg.all_reduce(t)

    def close(self) -> None:
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int) -> None:
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"bench_clocks_{os.getpid()}.csv"

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(name: str) -> float | None:
    """DRAM bytes per algorithmic byte of a tick, from the committed ncu summary."""
    p = ROOT / "profiles" / f"{name}.traffic"
    try:
        return float(p.read_text().split()[0])
    except (OSError, ValueError, IndexError):
        return None


# ---------------------------------------------------------------------------
# workload helpers
# ---------------------------------------------------------------------------
def build_workload(args):
    """The configuration's whole job (every rank builds the same seeded job)."""
    from ertm_b200 import workloads
    kw = {"nt": args.nt} if args.nt else {}
    return workloads.WORKLOADS[args.config](seed=0, **kw)


def shots_per_step(args) -> int:
    return int(args.shots or SHOTS_PER_STEP[args.config])


def step_shots(args, n_job: int, world: int, rank: int, k: int) -> list[int]:
    """Job shot indices this rank migrates in step k (warm-up steps
    included): the step takes the next shots_per_step·world shots of the job
    in order, wrapping around, and rank r takes its contiguous share."""
    s = shots_per_step(args)
    base = k * s * world + rank * s
    return [(base + j) % n_job for j in range(s)]


def job_config(wl, args, world: int) -> dict:
    g = wl.model.grid
    s = shots_per_step(args)
    return {"workload": wl.name, "config": args.config, "nx": g.nx, "nz": g.nz, "dx": g.dx, "nt": wl.nt,
            "dt": wl.dt, "engine": wl.engine, "modes": list(wl.modes), "condition": wl.condition,
            "separation": wl.separation, "shots_per_job": len(wl.sources), "shots_per_step": s * world,
            "receivers": wl.receivers.nrec, "components": list(wl.components), "q": wl.q or None,
            "checkpoint_mb": wl.checkpoint_mb, "accumulation": "fp64",
            "l2": "flushed between steps (256 MiB write); each step's inputs exceed L2 as well",
            "path": f"batched: a step's {s} shot(s) per GPU in lockstep ticks (form b), images stacked per step",
            "parallelism": f"shots sharded over {world} GPU(s), one float64 all-reduce of the stack per step"}


def imager_for(wl):
    from ertm_b200.workloads import imager_for as make
    return make(wl)


def synthesize(wl, solver, sources):
    """Shot records from the GPU forward model (untimed set-up)."""
    from ertm_b200.workloads import synthesize as make
    return make(wl, solver, sources)


def step_bytes(prop) -> float:
    """Algorithmic HBM bytes of one propagator step: each state array read and
    written once, each per-cell coefficient read once, CPML strips read and
    written (8 B per strip cell per term)."""
    info = prop.info()
    npad = info.nzp * info.nxp
    n_state = {"acoustic": 3, "elastic": 5, "viscoacoustic": 4 + getattr(prop, "n_mechanisms", 0)}[prop._engine]
    n_coef = {"acoustic": 3, "elastic": 5, "viscoacoustic": 3 + 2 * getattr(prop, "n_mechanisms", 0)}[prop._engine]
    _, _, _, _, (xl, xr, zt, zb) = prop._strips()
    nterm = len(prop._psi_terms) // 2
    strips = nterm * ((xl + xr) * info.nzp + (zt + zb) * info.nxp)
    return float(npad * (8 * n_state + 4 * n_coef) + 8 * strips)


# ---------------------------------------------------------------------------
# CPU oracle sample (baseline)
# ---------------------------------------------------------------------------
def cpu_sample(config: str, nt_sample: int, nt_override: int | None = None) -> dict:
    """Time the CPU oracle (NumPy restatement of the reference, single
    thread) migrating one shot of the workload for nt_sample steps."""
    import oracle as orc
    from ertm_b200 import workloads
    wl = workloads.WORKLOADS[config](seed=0, **({"nt": nt_override} if nt_override else {}))
    imager, solver = imager_for(wl)
    nrec = wl.receivers.nrec
    rng = np.random.default_rng(5)
    comps = {c: rng.normal(scale=1e-3, size=(nt_sample, nrec)).astype(np.float32) for c in wl.components}
    from types import SimpleNamespace
    sv = SimpleNamespace(**{k: getattr(solver, k) for k in ("dt", "order", "boundary", "dtype", "engine", "npml")},
                         nt=nt_sample)
    q = None
    if wl.q:
        q = SimpleNamespace(enabled=True, f_ref=wl.q["f_ref"], n_mechanisms=wl.q["n_mechanisms"], band_ratio=1.5,
                            compensation=True, alpha_c=wl.q["alpha_c"], amplitude_cap=wl.q["amplitude_cap"],
                            lowpass_interval=wl.q["lowpass_interval"], f_max=wl.q["f_max"],
                            gain_budget_db=wl.q["gain_budget_db"])
    t0 = time.perf_counter()
    orc.migrate(comps, wl.dt, wl.sources[0], wl.receivers, wl.model, sv, imager.config, q)
    return {"secs": time.perf_counter() - t0, "nt_sample": nt_sample, "nt": wl.nt, "cells": wl.cells,
            "migrates_per_shot": len(wl.modes)}      # the reference runs one RTMImager per imaging mode


def per_shot_seconds(short: list[dict], long: list[dict]) -> dict:
    """Split sample timings of two lengths into set-up and per-step cost and
    extrapolate one whole shot: setup + per_step · nt, times the migrates a
    shot needs.  Steps of the samples that never reach a periodic low-pass
    (every 20th backward step from step 40) leave its FFT cost out, which
    favours the CPU."""
    n1, n2 = short[0]["nt_sample"], long[0]["nt_sample"]
    t1 = statistics.mean(r["secs"] for r in short)
    t2 = statistics.mean(r["secs"] for r in long)
    per_step = max(t2 - t1, 1e-9) / (n2 - n1)
    setup = max(t1 - n1 * per_step, 0.0)
    r = long[0]
    return {"per_shot_s": (setup + per_step * r["nt"]) * r["migrates_per_shot"], "setup_s": setup,
            "per_step_s": per_step, "n1": n1, "n2": n2, "nt": r["nt"], "cells": r["cells"],
            "migrates_per_shot": r["migrates_per_shot"]}


def _cpu_worker(task):
    sys.path[:0] = [str(ROOT), str(ROOT / "challenge-cup_b200")]
    return cpu_sample(*task)


def run_reference(args, dist: Dist) -> None:
    """The reference's CPU implementation of the path (the NumPy oracle port:
    the reference is pure Python) on every host core of rank 0's machine."""
    if dist.rank != 0:
        return
    import multiprocessing as mp
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    cores = os.cpu_count() or 1
    n1, n2 = 4, 16
    ctx = mp.get_context("spawn")
    walls, shorts, longs = [], [], []
    with ctx.Pool(cores) as pool:
        for i in range(args.warmup + args.steps):
            tasks = [(args.config, n1 if c % 2 == 0 else n2, args.nt) for c in range(cores)]
            t0 = time.perf_counter()
            res = pool.map(_cpu_worker, tasks)
            if i >= args.warmup:
                walls.append(time.perf_counter() - t0)
                shorts += [r for r in res if r["nt_sample"] == n1]
                longs += [r for r in res if r["nt_sample"] == n2]
    est = per_shot_seconds(shorts, longs or shorts)
    value = cores / est["per_shot_s"]
    sample = (f"{cores} spawned single-threaded processes per step, each migrating one shot of the workload for "
              f"{n1} or {n2} of {est['nt']} steps with the NumPy oracle; set-up ({est['setup_s']:.2f} s) and "
              f"per-step cost ({est['per_step_s'] * 1e3:.0f} ms) separated from the two lengths and extrapolated "
              f"to the whole shot, x{est['migrates_per_shot']} migrates per shot (one per imaging mode)")
    wl = build_workload(args)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "shots/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(walls) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": job_config(wl, args, args.gpus),
            "gcell_updates_per_s": value * 3 * est["nt"] * est["cells"] * est["migrates_per_shot"] / 1e9,
            "cpu_baseline": {"value": value, "unit": "shots/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving (form c)
# ---------------------------------------------------------------------------
SERVE_SCALES = {
    # seconds: grids 256x256..1024x512, nt 500-2000, 1-4 shots
    "short": dict(max_scale=(4.0, 2.0), nt_range=(500, 2000), max_shots=4),
    # the serving configuration: grids 256x256..4096x2048, nt 1000-8000, 1-16 shots
    "full": dict(max_scale=(16.0, 8.0), nt_range=(1000, 8000), max_shots=16),
}


def serving_run(n_jobs: int, scale: str = "short", fractions=(0.5, 0.8)) -> dict:
    """The serving loop on a stream of mixed jobs: once with every job queued
    at t=0 (saturation), then with Poisson arrivals at the given fractions of
    the saturated job rate; per-shot latency = shot completion - job
    submission.  Jobs are admitted by their device footprint under the
    server's budget (170 GB, at most 90 % of free memory)."""
    from ertm_b200 import workloads
    from ertm_b200.serving import RTMServer, percentile
    spec = SERVE_SCALES[scale]
    jobs = workloads.serving_jobs(seed=1, n_jobs=n_jobs, **spec)
    n_shots = sum(len(j.shots) for j in jobs)
    cells = sum(3 * j.model.grid.nx * j.model.grid.nz * j.imager.solver_config.nt * len(j.shots) for j in jobs)

    def run(arrivals):
        with RTMServer() as srv:
            t0 = time.perf_counter()
            futs = []
            for job, at in zip(jobs, arrivals):
                delay = t0 + at - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futs.append(srv.submit(job))
            res = [f.result() for f in futs]
            wall = max(r.finished for r in res) - t0
        lat = [x for r in res for x in r.shot_latencies]
        return {"shots_per_s": n_shots / wall, "wall_s": wall, "shot_latency_p50_s": percentile(lat, 50),
                "shot_latency_p99_s": percentile(lat, 99),
                "job_latency_p50_s": percentile([r.latency for r in res], 50),
                "job_latency_p99_s": percentile([r.latency for r in res], 99),
                "peak_active_shots": srv.stats["peak_active"], "peak_bytes": srv.stats["peak_bytes"]}

    def plain() -> dict:
        """The same jobs through the plain one-shot path: every shot migrated
        alone (host records in, host images out), then each job stacked."""
        from ertm_b200.stacking import stack_images
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for job in jobs:
            modes = tuple(job.modes or (job.imager.config.mode,))
            per = [job.imager.migrate_modes(s, job.model, modes=modes) for s in job.shots]
            if job.stack:
                for k in range(len(modes)):
                    stack_images([r[k] for r in per])
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        return {"shots_per_s": n_shots / wall, "wall_s": wall}

    # warm-up (division checks, FFT plans, memory pool): the whole stream when
    # it takes seconds, its first jobs when it takes minutes
    run([0.0] * (len(jobs) if scale == "short" else min(len(jobs), 3)))
    sat = run([0.0] * len(jobs))
    job_rate = len(jobs) / sat["wall_s"]
    plain_line = plain()
    rng = np.random.default_rng(7)
    sx, sz = spec["max_scale"]
    out = {"workload": (f"{n_jobs} jobs, engine uniform over acoustic/elastic/viscoacoustic, grid 256x256.."
                        f"{int(256 * sx)}x{int(256 * sz)} log-uniform at 5-10 m, nt {spec['nt_range'][0]}-"
                        f"{spec['nt_range'][1]}, 1-{spec['max_shots']} shots, normalized, seeded noise records"),
           "scale": scale,
           "shots": n_shots, "gcell_updates": cells / 1e9, "saturation": sat,
           "saturation_gcell_updates_per_s": cells / sat["wall_s"] / 1e9,
           "plain": plain_line, "served_over_plain": sat["shots_per_s"] / plain_line["shots_per_s"]}
    for frac in fractions:
        lam = frac * job_rate
        arrivals = np.cumsum(rng.exponential(1.0 / lam, len(jobs)))
        out[f"poisson_{int(frac * 100)}pct"] = {"lambda_jobs_per_s": lam, **run(list(arrivals))}
    return out


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def adjacent_rows_run(wl, peak: float, cpu: bool) -> dict:
    """The steps either side of the path, on one job's data (all shots of the
    workload), device-resident, each call timed with CUDA events after an L2
    flush: record preprocessing (sinc resampling from a 1 ms field record,
    direct-wave mute, end taper), the data-domain Q filter, SEG-Y decoding of
    the job's records, per-shot image post-processing and the stack.  Bytes
    are algorithmic (inputs read once, outputs written once); ``cpu_s`` is the
    oracle on the same call (single thread), where ``cpu`` is set."""
    import ctypes as C

    import torch

    from ertm_b200 import _lib, segy
    from ertm_b200.preprocess import resample_weights
    from oracle import ertm_oracle as orc

    L = _lib.lib()
    g = wl.model.grid
    n_shots, ncomp, nt, nrec = len(wl.sources), len(wl.components), wl.nt, wl.receivers.nrec
    ntr = n_shots * ncomp * nrec                      # every trace of the job side by side
    npix = g.nx * g.nz
    gen = torch.Generator(device="cuda").manual_seed(5)
    rec = torch.randn((nt, ntr), generator=gen, device="cuda", dtype=torch.float32)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def timed(call, reps=5):
        for _ in range(2):
            call()
        ms = []
        for _ in range(reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            call()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    def cpu_time(fn):
        if not cpu:
            return None
        t0 = time.perf_counter()
        fn()
        return time.perf_counter() - t0

    rows = {}

    def add(name, ms, nbytes, what, cpu_s=None):
        gbs = nbytes / (ms * 1e-3) / 1e9
        rows[name] = {"ms": ms, "bytes": int(nbytes), "gbs": gbs, "frac": gbs / peak, "what": what, "cpu_s": cpu_s}

    # sinc resampling: a 1 ms record of the same duration to the propagation dt
    n_in = int(np.floor((nt - 1) * wl.dt / 1e-3)) + 1
    w, off0 = resample_weights(n_in, 1e-3, wl.dt)
    n_out = w.shape[0]
    rin = torch.randn((n_in, ntr), generator=gen, device="cuda", dtype=torch.float32)
    rout = torch.empty((n_out, ntr), device="cuda", dtype=torch.float32)
    wd, od = torch.from_numpy(w).cuda(), torch.from_numpy(off0).cuda()
    ms = timed(lambda: _lib.check(L.ertm_resample(rin.data_ptr(), n_in, ntr, wd.data_ptr(), od.data_ptr(),
                                                  w.shape[1], n_out, rout.data_ptr(), None), "resample"))
    host_in = rin[:, :nrec].cpu().numpy()
    add("resample", ms, 4 * (n_in + n_out) * ntr + w.nbytes + off0.nbytes,
        f"sinc resampling 1 ms -> {wl.dt * 1e3:.4f} ms, {n_in}->{n_out} samples x {ntr} traces",
        None if not cpu else cpu_time(lambda: orc.resample_sinc(host_in, 1e-3, wl.dt)) * (ntr / nrec))

    # direct-wave mute and end taper over every trace of the job
    t = torch.arange(nt, device="cuda", dtype=torch.float64) * wl.dt
    start = torch.linspace(0.05, 0.4, ntr, device="cuda", dtype=torch.float64)
    end = start + 0.02
    out = torch.empty_like(rec)
    ms = timed(lambda: _lib.check(L.ertm_mute(rec.data_ptr(), nt, ntr, t.data_ptr(), start.data_ptr(),
                                              end.data_ptr(), out.data_ptr(), None), "mute"))
    add("mute", ms, 8 * nt * ntr + 8 * nt + 16 * ntr, f"cosine direct-wave mute, {nt} x {ntr}")
    wt = max(int(0.05 * nt), 1)
    ramp = torch.from_numpy(0.5 - 0.5 * np.cos(np.pi * (np.arange(wt) + 0.5) / wt)).cuda()
    ms = timed(lambda: _lib.check(L.ertm_taper(rec.data_ptr(), nt, ntr, ramp.data_ptr(), wt, out.data_ptr(), None),
                                  "taper"))
    host = rec[:, :nrec].cpu().numpy()
    add("taper", ms, 8 * nt * ntr + 8 * wt, f"end taper 5%, {nt} x {ntr}",
        None if not cpu else cpu_time(lambda: orc.taper_ends(host, 0.05)) * (ntr / nrec))

    # data-domain Q filter on the job's pressure records (float64, nperseg 128, 50 % overlap)
    nq = n_shots * nrec
    q_in = rec[:, :nq].double().contiguous()
    q_out = torch.empty_like(q_in)
    Lf, hop = 128, 64
    S = len(range(0, nt, hop)) - sum(1 for s in range(0, nt, hop) if min(s + Lf, nt) - s < 4)
    freqs = np.fft.rfftfreq(Lf, d=wl.dt)
    resp = np.stack([orc.q_attenuation_response(freqs, (s * hop + 0.5 * Lf) * wl.dt, 60.0, 30.0)
                     for s in range(S)])
    resp_d = torch.from_numpy(np.ascontiguousarray(resp).view(np.float64)).cuda()
    win = torch.from_numpy(np.hanning(Lf)).cuda()
    ms = timed(lambda: _lib.check(L.ertm_stft_filter(q_in.data_ptr(), nt, nq, Lf, hop, S, win.data_ptr(),
                                                     resp_d.data_ptr(), q_out.data_ptr(), None), "stft"))
    qh = q_in[:, :nrec].cpu().numpy()
    add("q_filter", ms, 16 * nt * nq + resp.nbytes, f"STFT Q filter, {nt} x {nq} float64, {S} frames of {Lf}",
        None if not cpu else cpu_time(lambda: orc.stft_filter(
            qh, wl.dt, lambda tc, f: orc.q_attenuation_response(f, max(tc, 1e-6), 60.0, 30.0))) * (nq / nrec))

    # SEG-Y: the job's records as one IEEE file section, decoded into per-record (nt, nrec) blocks
    tb = 240 + 4 * nt
    section = torch.zeros(ntr * tb, dtype=torch.uint8, device="cuda")
    hdr = np.zeros(ntr, dtype=segy.TRACE_DTYPE)
    hdr["TraceNumber"] = np.arange(1, ntr + 1)
    hdr["TRACE_SAMPLE_COUNT"] = nt
    hb = hdr.view(np.uint8)
    _lib.check(L.ertm_segy_encode(rec.data_ptr(), nt, ntr, 5, hb.ctypes.data, section.data_ptr(), None), "encode")
    perm = np.arange(ntr).reshape(-1, nrec)
    order = np.ascontiguousarray(perm.reshape(-1), dtype=np.int32)
    dest = np.ascontiguousarray((np.arange(ntr) // nrec) * nt * nrec + np.arange(ntr) % nrec, dtype=np.int64)
    width = np.full(ntr, nrec, dtype=np.int32)
    dec = torch.empty(nt * ntr, dtype=torch.float32, device="cuda")
    ms = timed(lambda: _lib.check(L.ertm_segy_decode(section.data_ptr(), ntr, nt, 5, ntr, order.ctypes.data,
                                                     dest.ctypes.data, width.ctypes.data, dec.data_ptr(),
                                                     dec.numel(), None), "decode"))
    blob = None
    if cpu:
        blob = orc.segy_bytes(host, [{"TRACE_SAMPLE_COUNT": nt}] * nrec, 1000, 5, "")
    add("segy_decode", ms, ntr * tb + 4 * nt * ntr + 16 * ntr,
        f"SEG-Y IEEE decode + transpose, {ntr} traces of {nt} samples into {ntr // nrec} records",
        None if not cpu else cpu_time(lambda: orc.segy_parse(blob)) * (ntr / nrec))

    # per-shot post-processing (normalisation by illumination, Laplacian, mask) and the stack
    num = torch.randn((npix,), generator=gen, device="cuda", dtype=torch.float64)
    ill = torch.rand((npix,), generator=gen, device="cuda", dtype=torch.float64) + 0.1
    img = torch.empty((npix,), device="cuda", dtype=torch.float32)
    ms = timed(lambda: _lib.check(L.ertm_postprocess(g.nz, g.nx, float(g.dx), float(g.dz), num.data_ptr(),
                                                     ill.data_ptr(), None, 1, 0, 1e-6, 1, 1.0, 20, 1,
                                                     img.data_ptr(), None), "postprocess"))
    nh, ih = num.view(g.nz, g.nx).cpu().numpy(), ill.view(g.nz, g.nx).cpu().numpy()
    add("postprocess", ms, 16 * npix + 4 * npix, f"illumination normalisation + Laplacian + PML mask, {g.nz} x {g.nx}",
        None if not cpu else cpu_time(lambda: orc.postprocess(nh / (ih + 1e-6), g.dx, g.dz, laplacian_on=True,
                                                              lowpass_fraction=1.0, npml=20, boundary="cpml")))
    imgs = torch.randn((n_shots, npix), generator=gen, device="cuda", dtype=torch.float32)
    acc = torch.zeros((npix,), device="cuda", dtype=torch.float64)
    fin = torch.empty((npix,), device="cuda", dtype=torch.float32)
    ptrs = (C.c_void_p * n_shots)(*[imgs[i].data_ptr() for i in range(n_shots)])

    def stack():
        acc.zero_()
        _lib.check(L.ertm_stack_partial(n_shots, npix, C.cast(ptrs, C.c_void_p), 1, acc.data_ptr(), None), "stack")
        _lib.check(L.ertm_stack_finish(npix, acc.data_ptr(), n_shots, fin.data_ptr(), None), "finish")
    ms = timed(stack)
    ih = [im.view(g.nz, g.nx).cpu().numpy() for im in imgs]
    add("stack", ms, n_shots * 4 * npix + 8 * npix + 4 * npix,
        f"per-shot max-normalised float64 stack of {n_shots} images {g.nz} x {g.nx}",
        None if not cpu else cpu_time(lambda: orc.stack_images(ih, normalize=True)))
    return rows


def uneven_run(n_shots: int) -> dict:
    """A bounded sample of the uneven batch (the 256-shot configuration: 4
    seeded models of 501×301 … 2401×1201, acoustic or elastic, nt 1500-6000,
    10-30 Hz): its first n_shots shots migrated in lockstep ticks (memory
    grouped) and one at a time through the plain path; images compared."""
    import torch

    from ertm_b200 import workloads
    from ertm_b200.batch import DeviceShot, migrate_device_items
    from ertm_b200.imaging import ShotMigrator
    from ertm_b200.propagation import source_wavelet
    wls = workloads.uneven_batch(seed=0, n_shots=256)[:n_shots]
    items, plain_in, cells = [], [], 0
    for wl in wls:
        imager, solver = imager_for(wl)
        shot = synthesize(wl, solver, wl.sources)[0]
        names = list(wl.components)
        rec = torch.from_numpy(np.stack([shot.components[n] for n in names])).cuda()
        w = source_wavelet(wl.sources[0], wl.dt, wl.nt)
        items.append(DeviceShot(ShotMigrator(imager, wl.model), wl.sources[0], wl.receivers, rec, names, w,
                                tuple(wl.modes)))
        plain_in.append(ShotMigrator(imager, wl.model))
        cells += 3 * wl.nt * wl.cells
    torch.cuda.synchronize()

    def batched():
        return migrate_device_items(items)

    def plain():
        return [pm.migrate_device(it.source, it.receivers, it.record, it.names, it.wavelet, modes=it.modes)
                for pm, it in zip(plain_in, items)]

    out = {}
    for name, fn in (("batched", batched), ("plain", plain)):
        fn()                                   # warm-up: tables, division checks, plans
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        imgs = fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"ms": ms, "shots_per_s": len(items) / (ms / 1e3), "gcell_updates_per_s": cells / (ms / 1e3) / 1e9,
                     "images": imgs}
    same = all(torch.equal(a, b) for a, b in zip(out["batched"].pop("images"), out["plain"].pop("images")))
    kinds = {}
    for wl in wls:
        key = f"{wl.engine} {wl.model.grid.nx}x{wl.model.grid.nz}"
        kinds[key] = kinds.get(key, 0) + 1
    return {"workload": f"first {len(items)} of the 256 uneven shots (seeded): {kinds}, nt "
                        f"{min(w.nt for w in wls)}-{max(w.nt for w in wls)}",
            "gcell_updates": cells / 1e9, **out,
            "batched_over_plain": out["batched"]["shots_per_s"] / out["plain"]["shots_per_s"],
            "batched_equals_plain": bool(same)}


def run_ours(args, dist: Dist) -> None:
    import ctypes as C

    import torch

    from ertm_b200 import _lib
    from ertm_b200.batch import DeviceShot, migrate_device_items
    from ertm_b200.imaging import ShotMigrator
    from ertm_b200.parallel import ShotParallelMigrator, plan_shards, reduce_partial_sums, shot_cost
    from ertm_b200.propagation import source_wavelet
    from ertm_b200.types import ShotRecord

    dev = dist.local
    torch.cuda.set_device(dev)
    L = _lib.lib(dev)
    wl = build_workload(args)
    imager, solver = imager_for(wl)
    g = wl.model.grid
    n_job = len(wl.sources)
    S = shots_per_step(args)
    per_step = S * dist.world                       # shots of one step over all ranks
    n_all = args.warmup + args.steps
    plan = [step_shots(args, n_job, dist.world, dist.rank, k) for k in range(n_all)]
    used = sorted({i for st in plan for i in st})
    names = list(wl.components)
    n_modes = len(wl.modes)
    npix = g.nx * g.nz
    # the shots' records from the GPU forward model (untimed set-up), kept on the device
    recs = dict(zip(used, synthesize(wl, solver, [wl.sources[i] for i in used])))
    rec_dev = {i: torch.from_numpy(np.stack([recs[i].components[n] for n in names])).cuda() for i in used}
    wavelets = {i: source_wavelet(wl.sources[i], wl.dt, wl.nt) for i in used}
    plain_mig = ShotMigrator(imager, wl.model)                       # one propagator pair, reused
    batch_migs = [ShotMigrator(imager, wl.model) for _ in range(S)]  # one pair per shot of a step
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > 126 MB L2
    partial = torch.empty((n_modes, g.nz, g.nx), dtype=torch.float64, device="cuda")

    def stack(imgs, out):
        """This rank's float64 partial stack, the step's one all-reduce, finish."""
        partial.zero_()
        for k in range(n_modes):
            ptrs = (C.c_void_p * len(imgs))(*[im[k].data_ptr() for im in imgs])
            _lib.check(L.ertm_stack_partial(len(imgs), npix, C.cast(ptrs, C.c_void_p), int(per_step > 1),
                                            partial[k].data_ptr(), None), "stack partial")
        if dist.world > 1:
            reduce_partial_sums(partial)
        for k in range(n_modes):
            _lib.check(L.ertm_stack_finish(npix, partial[k].data_ptr(), per_step, out[k].data_ptr(), None),
                       "stack finish")
        return out

    out_plain = torch.empty((n_modes, g.nz, g.nx), dtype=torch.float32, device="cuda")
    out_batch = torch.empty_like(out_plain)

    def plain_step(k):
        imgs = [plain_mig.migrate_device(wl.sources[i], wl.receivers, rec_dev[i], names, wavelets[i],
                                         modes=wl.modes) for i in plan[k]]
        return stack(imgs, out_plain)

    def batch_step(k):
        items = [DeviceShot(batch_migs[j], wl.sources[i], wl.receivers, rec_dev[i], names, wavelets[i],
                            tuple(wl.modes)) for j, i in enumerate(plan[k])]
        return stack(migrate_device_items(items), out_batch)

    def timed(step, warm: list[int], steps: list[int], profile: bool):
        for k in warm:
            step(k)
        torch.cuda.synchronize()
        if profile:
            _lib.check(L.ertm_profile_stencil(1, 4), "profile")
        launches0 = L.ertm_launch_count()
        times, first = [], None
        dist.barrier()
        torch.cuda.synchronize()
        for k in steps:
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = step(k)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            if first is None:
                first = out.clone()
        dist.barrier()
        torch.cuda.synchronize()
        return times, int(L.ertm_launch_count() - launches0), first

    timed_steps = list(range(args.warmup, n_all))
    # plain one-shot path (reported beside the batched form) on the first timed steps' shots
    n_plain = max(1, min(args.plain_steps, args.steps))
    plain_times, _, plain_first = timed(plain_step, [0], timed_steps[:n_plain], False)
    clocks = Clocks(dev)
    clocks.start()
    times, launches, batch_first = timed(batch_step, list(range(args.warmup)), timed_steps, True)
    clk = clocks.stop()
    tot, cnt, byt = C.c_double(), C.c_int64(), C.c_double()
    _lib.check(L.ertm_profile_read(C.byref(tot), C.byref(cnt), C.byref(byt)), "profile read")
    _lib.check(L.ertm_profile_stencil(0, 1), "profile off")
    same = bool(torch.equal(plain_first, batch_first))

    total_ms = dist.max(float(sum(times)))
    plain_ms = dist.max(float(sum(plain_times)))
    value = per_step * args.steps / (total_ms / 1e3)
    plain_value = per_step * n_plain / (plain_ms / 1e3)
    cells_per_shot = 3 * wl.nt * wl.cells

    # end to end through the public API: every rank is handed the step's
    # shots as host records (pinned), migrates its shard and gets the stacked
    # host images back; host<->device copies are inside the timed region
    e2e_times, h2d, d2h = [], 0, 0
    spm = ShotParallelMigrator(imager, group=None)     # keeps its propagator pairs between calls
    e2e_steps = timed_steps[: max(0, args.e2e_steps)]
    for n_call, k in enumerate(e2e_steps[:1] + e2e_steps):   # the first call (untimed) builds the pairs
        glob = [(k * per_step + j) % n_job for j in range(per_step)]
        costs = [shot_cost(g.nx, g.nz, wl.nt, wl.engine)] * per_step
        mine = set(plan_shards(costs, dist.world)[dist.rank])
        host_shots = []
        for j, i in enumerate(glob):
            if j in mine:
                if i not in recs:
                    recs[i] = synthesize(wl, solver, [wl.sources[i]])[0]
                r = recs[i]
                comps = {n: torch.from_numpy(r.components[n]).pin_memory().numpy() for n in names}
            else:      # another rank's shot: only its shape enters the shard plan here
                comps = {n: np.zeros((wl.nt, wl.receivers.nrec), np.float32) for n in names}
            host_shots.append(ShotRecord(data=comps[names[0]], dt=wl.dt, t=np.arange(wl.nt) * wl.dt,
                                         receivers=wl.receivers, source=wl.sources[i], components=comps))
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        stacked = spm.migrate_job(host_shots, wl.model, modes=wl.modes)
        torch.cuda.synchronize()
        if n_call:
            e2e_times.append(time.perf_counter() - t0)
        assert all(np.isfinite(r.image).all() for r in stacked)
    comp_bytes = len(names) * wl.nt * wl.receivers.nrec * 4
    model_bytes = 3 * npix * 4 * 2                      # vp, vs, rho per propagator, two propagators
    # summed over the step's ranks: records, models and wavelets in; the stacked images out
    # (per-shot accumulators are created, post-processed and stacked on the device)
    h2d = per_step * (comp_bytes + model_bytes + wl.nt * 4)
    d2h = dist.world * n_modes * npix * 4
    e2e_s = dist.max(statistics.mean(e2e_times)) if e2e_times else float("nan")
    e2e_value = per_step / e2e_s

    tuned = L.ertm_autotune_report().decode().strip().splitlines()   # the batched job's shapes
    uneven = uneven_run(args.uneven_shots) if dist.world == 1 and args.uneven_shots > 0 else None
    serving = None
    if dist.world == 1 and args.serve_jobs > 0:
        fr = (0.5, 0.8) if args.serve_scale == "short" else (0.25, 0.5, 0.75, 1.0, 1.25)
        serving = serving_run(args.serve_jobs, args.serve_scale, fr)

    peak, peak_kind = measured_hbm_peak()
    adjacent = None
    if dist.world == 1 and not args.no_adjacent:
        adjacent = adjacent_rows_run(wl, peak, cpu=not args.no_cpu_baseline)
    step_ms = float(tot.value) / max(int(cnt.value), 1)
    achieved = float(byt.value) / (float(tot.value) * 1e-3) / 1e9 if tot.value > 0 else 0.0
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        n2 = max(args.cpu_sample_steps, 8)
        n1 = max(n2 // 3, 4)
        est = per_shot_seconds([cpu_sample(args.config, n1, args.nt)], [cpu_sample(args.config, n2, args.nt)])
        cpu = {"value": 1.0 / est["per_shot_s"], "unit": "shots/s", "cores": 1, "kind": "port",
               "sample": (f"one shot of the workload, {n1} and {n2} of {est['nt']} steps of the NumPy oracle migrate "
                          f"on one core; set-up ({est['setup_s']:.2f} s) and per-step cost "
                          f"({est['per_step_s'] * 1e3:.0f} ms) separated from the two lengths, extrapolated to the "
                          f"whole shot, x{est['migrates_per_shot']} for one migrate per imaging mode")}
    traffic_ratio = committed_traffic(f"{wl.engine}_step")
    line = {
        "metric": METRIC, "value": value, "unit": "shots/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded layered model; records from the GPU forward model",
        "config": job_config(wl, args, dist.world),
        "gcell_updates_per_s": cells_per_shot * per_step * args.steps / (total_ms / 1e3) / 1e9,
        "plain": {"value": plain_value, "unit": "shots/s", "ms_per_step": plain_ms / n_plain, "steps": n_plain,
                  "gcell_updates_per_s": cells_per_shot * per_step * n_plain / (plain_ms / 1e3) / 1e9,
                  "path": "one shot at a time, same kernels, same shots as the first timed batched steps"},
        "batched_over_plain": value / plain_value,
        "batched_equals_plain": same,
        "e2e": {"value": e2e_value, "unit": "shots/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "steps": len(e2e_times), "path": "ShotParallelMigrator.migrate_job: host records in, stacked host "
                                                 "images out, one step's shots per call; one untimed call before "
                                                 "builds the propagator pairs the later calls reuse"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (None if traffic_ratio is None else
                                 traffic_ratio * float(byt.value) / max(int(cnt.value), 1)),
                     "traffic_note": ("DRAM bytes per tick: the DRAM/algorithmic ratio ncu measured on a captured "
                                      f"tick of this configuration (profiles/{wl.engine}_step.traffic) times this "
                                      "run's algorithmic bytes per tick"),
                     "kernel": f"{wl.engine} velocity + stress launches of a batched tick (imaging epilogue fused)",
                     "bytes_definition": "per propagator step: Npad*(8*n_state + 4*n_coef) + 8*CPML strip cells*terms;"
                                         " per fused imaging epilogue: 16 B per accumulator, 4 B per replayed field",
                     "bytes_per_tick": float(byt.value) / max(int(cnt.value), 1), "tick_us": step_ms * 1e3,
                     "timed_ticks": int(cnt.value), "peak_source": peak_kind},
        "cpu_baseline": cpu,
        "uneven": uneven,
        "serving": serving,
        "adjacent_rows": adjacent,
        "autotune": tuned,
        "stage_timeouts": int(L.ertm_stage_timeouts()),
        "clocks": clk,
        "gpu_launches": launches,
    }
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    args = parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args))
    # the reference arm is a CPU run on rank 0 alone: no process group, so the
    # other ranks exit at once instead of waiting for rank 0 in a collective
    dist = Dist(join=args.impl != "reference")
    try:
        if args.serving_only:
            import torch
            torch.cuda.set_device(dist.local)
            fr = (0.5, 0.8) if args.serve_scale == "short" else (0.25, 0.5, 0.75, 1.0, 1.25)
            clocks = Clocks(dist.local)
            clocks.start()
            out = serving_run(args.serve_jobs, args.serve_scale, fr)
            out["clocks"] = clocks.stop()
            if dist.rank == 0:
                print(json.dumps({"serving": out}), flush=True)
        elif args.impl == "reference":
            run_reference(args, dist)
        else:
            run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
