#!/usr/bin/env python
"""Benchmark of the B200 RTM hot path.

Default workload (one GPU): elastic P-SV borehole 4C RTM with PP and PS
imaging — 401×601 grid at 5 m, 8 surface shots, 100 well receivers, 4912
steps (1.5 s at the CFL dt), normalized condition, divcurl separation.  A
benchmark step migrates all shots of the job (PP and PS from one
forward/replay/backward pass per shot) and stacks them.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
    torchrun --nproc-per-node N bench.py --gpus N ...   (weak scaling: a job
        of 8·N shots sharded over the ranks; one NCCL all-reduce of the
        float64 stack per job)

One JSON line is printed by rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
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


def parse_args() -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", default="elastic4c")
    ap.add_argument("--nt", type=int, default=None, help="override the number of time steps (profiling runs)")
    ap.add_argument("--shots", type=int, default=None, help="override shots per rank")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=48)
    ap.add_argument("--serve-jobs", type=int, default=24, help="jobs in the serving run (0: no serving run)")
    ap.add_argument("--no-adjacent", action="store_true",
                    help="skip timing the steps either side of the path (preprocessing, Q filter, SEG-Y, stack)")
    return ap.parse_args()


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
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
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
def build_workload(args, world: int):
    """The job's workload: the configuration's shots per GPU times the world
    size (weak scaling), every rank building the same seeded job."""
    from ertm_b200 import workloads
    kw = {"nt": args.nt} if args.nt else {}
    make = workloads.WORKLOADS[args.config]
    wl = make(seed=0, **kw, **({"n_shots": args.shots} if args.shots else {}))
    if world > 1:
        wl = make(seed=0, n_shots=len(wl.sources) * world, **kw)
    return wl


def job_config(wl, args, world: int) -> dict:
    g = wl.model.grid
    return {"workload": wl.name, "config": args.config, "nx": g.nx, "nz": g.nz, "dx": g.dx, "nt": wl.nt,
            "dt": wl.dt, "engine": wl.engine, "modes": list(wl.modes), "condition": wl.condition,
            "separation": wl.separation, "shots_per_job": len(wl.sources), "receivers": wl.receivers.nrec,
            "components": list(wl.components), "accumulation": "fp64",
            "l2": "flushed between steps (256 MiB write)",
            "path": "batched: all shots of a rank in lockstep ticks (form b)",
            "parallelism": f"shots sharded over {world} GPU(s), one float64 all-reduce of the stack per job"}


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
def cpu_sample(config: str, nt_sample: int) -> dict:
    """Time the CPU oracle (NumPy restatement of the reference) migrating one
    shot of the workload for nt_sample steps; extrapolate to the full job."""
    import oracle as orc
    from ertm_b200 import workloads
    wl = workloads.WORKLOADS[config](seed=0)
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
    secs = time.perf_counter() - t0
    migrates_per_shot = len(wl.modes)      # the reference runs one RTMImager per mode
    per_shot = secs * (wl.nt / nt_sample) * migrates_per_shot
    return {"per_shot_s": per_shot, "sample_s": secs, "nt_sample": nt_sample, "nt": wl.nt,
            "migrates_per_shot": migrates_per_shot, "cells": wl.cells}


def _cpu_worker(args):
    config, nt_sample = args
    sys.path[:0] = [str(ROOT), str(ROOT / "challenge-cup_b200")]
    return cpu_sample(config, nt_sample)


def run_reference(args, dist: Dist) -> None:
    if dist.rank != 0:
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    nt_sample = max(8, args.cpu_sample_steps // 4)
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(cores) as pool:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(_cpu_worker, [(args.config, nt_sample)] * cores)
            if i >= args.warmup:
                times.append((time.perf_counter() - t0, res))
    wall = sum(t for t, _ in times) / len(times)
    per_shot = statistics.mean(r["per_shot_s"] for _, rs in times for r in rs)
    value = cores / per_shot
    cells = times[0][1][0]["cells"]
    nt = times[0][1][0]["nt"]
    sample = (f"{cores} spawned processes, each migrating one shot of the workload for {nt_sample} of {nt} "
              f"steps with the NumPy oracle; extrapolated linearly in steps, x{times[0][1][0]['migrates_per_shot']}"
              f" migrates per shot (one per imaging mode)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "shots/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": job_config(build_workload(args, dist.world), args, dist.world),
            "gcell_updates_per_s": value * 3 * nt * cells * times[0][1][0]["migrates_per_shot"] / 1e9,
            "cpu_baseline": {"value": value, "unit": "shots/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving (form c)
# ---------------------------------------------------------------------------
def serving_run(n_jobs: int) -> dict:
    """The serving loop on a stream of mixed jobs: once with every job queued
    at t=0 (saturation), then with Poisson arrivals at 50 % and 80 % of the
    saturated job rate; per-shot latency = shot completion - job submission."""
    from ertm_b200 import workloads
    from ertm_b200.serving import RTMServer, percentile
    spec = dict(max_scale=(4.0, 2.0), nt_range=(500, 2000), max_shots=4)
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

    run([0.0] * len(jobs))                      # warm-up (division checks, FFT plans, memory pool)
    sat = run([0.0] * len(jobs))
    job_rate = len(jobs) / sat["wall_s"]
    plain_line = plain()
    rng = np.random.default_rng(7)
    out = {"workload": (f"{n_jobs} jobs, engine uniform over acoustic/elastic/viscoacoustic, grid 256x256..1024x512 "
                        f"log-uniform at 5-10 m, nt 500-2000, 1-4 shots, normalized, seeded noise records"),
           "shots": n_shots, "gcell_updates": cells / 1e9, "saturation": sat,
           "saturation_gcell_updates_per_s": cells / sat["wall_s"] / 1e9,
           "plain": plain_line, "served_over_plain": sat["shots_per_s"] / plain_line["shots_per_s"]}
    for frac in (0.5, 0.8):
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


def run_ours(args, dist: Dist) -> None:
    import ctypes as C

    import torch

    from ertm_b200 import _lib
    from ertm_b200.batch import migrate_device_batch
    from ertm_b200.imaging import ShotMigrator
    from ertm_b200.parallel import ShotParallelMigrator, plan_shards, reduce_partial_sums, shot_cost
    from ertm_b200.propagation import source_wavelet
    from ertm_b200.types import ShotRecord

    dev = dist.local
    torch.cuda.set_device(dev)
    L = _lib.lib(dev)
    wl = build_workload(args, dist.world)
    imager, solver = imager_for(wl)
    g = wl.model.grid
    n_total = len(wl.sources)
    mine = plan_shards([shot_cost(g.nx, g.nz, wl.nt, wl.engine)] * n_total, dist.world)[dist.rank]
    sources = [wl.sources[i] for i in mine]
    shots = synthesize(wl, solver, sources)
    names = list(wl.components)
    rec_dev = [torch.from_numpy(np.stack([s.components[n] for n in names])).cuda() for s in shots]
    wavelets = [source_wavelet(s, wl.dt, wl.nt) for s in sources]
    n_modes = len(wl.modes)
    n_shots = len(sources)
    npix = g.nx * g.nz
    plain_mig = ShotMigrator(imager, wl.model)                       # one propagator pair, reused
    batch_migs = [ShotMigrator(imager, wl.model) for _ in range(n_shots)]  # one pair per shot
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > 126 MB L2
    partial = torch.empty((n_modes, g.nz, g.nx), dtype=torch.float64, device="cuda")

    def stack(imgs, out):
        """This rank's float64 partial stack, the job's one all-reduce, finish."""
        partial.zero_()
        for k in range(n_modes):
            ptrs = (C.c_void_p * len(imgs))(*[im[k].data_ptr() for im in imgs])
            _lib.check(L.ertm_stack_partial(len(imgs), npix, C.cast(ptrs, C.c_void_p), int(n_total > 1),
                                            partial[k].data_ptr(), None), "stack partial")
        if dist.world > 1:
            reduce_partial_sums(partial)
        for k in range(n_modes):
            _lib.check(L.ertm_stack_finish(npix, partial[k].data_ptr(), n_total, out[k].data_ptr(), None),
                       "stack finish")
        return out

    out_plain = torch.empty((n_modes, g.nz, g.nx), dtype=torch.float32, device="cuda")
    out_batch = torch.empty_like(out_plain)

    def plain_job():
        imgs = [plain_mig.migrate_device(src, wl.receivers, rec_dev[i], names, wavelets[i], modes=wl.modes)
                for i, src in enumerate(sources)]
        return stack(imgs, out_plain)

    def batch_job():
        imgs = migrate_device_batch(imager, batch_migs, sources, [wl.receivers] * n_shots, rec_dev, names,
                                    wavelets, modes=wl.modes)
        return stack(imgs, out_batch)

    def timed(job, steps, profile: bool):
        for _ in range(args.warmup):
            job()
        torch.cuda.synchronize()
        if profile:
            _lib.check(L.ertm_profile_stencil(1, 4), "profile")
        launches0 = L.ertm_launch_count()
        times = []
        dist.barrier()
        torch.cuda.synchronize()
        for _ in range(steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            job()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        dist.barrier()
        torch.cuda.synchronize()
        return times, int(L.ertm_launch_count() - launches0)

    # plain one-shot path (reported beside the batched form)
    plain_times, _ = timed(plain_job, args.steps, False)
    clocks = Clocks(dev)
    clocks.start()
    times, launches = timed(batch_job, args.steps, True)
    clk = clocks.stop()
    tot, cnt, byt = C.c_double(), C.c_int64(), C.c_double()
    _lib.check(L.ertm_profile_read(C.byref(tot), C.byref(cnt), C.byref(byt)), "profile read")
    _lib.check(L.ertm_profile_stencil(0, 1), "profile off")
    same = bool(torch.equal(out_plain, out_batch))

    total_ms = dist.max(float(sum(times)))
    plain_ms = dist.max(float(sum(plain_times)))
    shots_total = n_total * args.steps
    value = shots_total / (total_ms / 1e3)
    plain_value = shots_total / (plain_ms / 1e3)
    cell_updates = 3 * wl.nt * wl.cells * shots_total

    # end to end through the public API: every rank is handed the whole job as
    # host shot records (pinned), migrates its shard and gets the stacked host
    # images back; host<->device copies are inside the timed region
    pinned = [{n: torch.from_numpy(s.components[n]).pin_memory().numpy() for n in names} for s in shots]
    host_shots = [None] * n_total
    for j, i in enumerate(mine):
        s = shots[j]
        host_shots[i] = ShotRecord(data=pinned[j][names[0]], dt=s.dt, t=s.t, receivers=s.receivers, source=s.source,
                                   components=pinned[j])
    for i in range(n_total):        # other ranks' shots: only their shape enters the shard plan here
        if host_shots[i] is None:
            host_shots[i] = ShotRecord(data=np.zeros((wl.nt, wl.receivers.nrec), np.float32), dt=wl.dt,
                                       t=np.arange(wl.nt) * wl.dt, receivers=wl.receivers, source=wl.sources[i],
                                       components={n: np.zeros((wl.nt, wl.receivers.nrec), np.float32)
                                                   for n in names})
    spm = ShotParallelMigrator(imager, group=None)
    e2e_times = []
    for _ in range(args.e2e_steps):
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        stacked = spm.migrate_job(host_shots, wl.model, modes=wl.modes)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        assert all(np.isfinite(r.image).all() for r in stacked)
    comp_bytes = len(names) * wl.nt * wl.receivers.nrec * 4
    model_bytes = 3 * npix * 4 * 2                      # vp, vs, rho per propagator, two propagators
    # summed over the job's ranks: records, models and wavelets in; per-shot images and the stack out
    # (accumulators are created, post-processed and stacked on the device)
    h2d = n_total * (comp_bytes + model_bytes + wl.nt * 4)
    d2h = n_total * n_modes * npix * 4 + dist.world * n_modes * npix * 4
    e2e_s = dist.max(statistics.mean(e2e_times)) if e2e_times else float("nan")
    e2e_value = n_total / e2e_s

    tuned = L.ertm_autotune_report().decode().strip().splitlines()   # the batched job's shapes
    serving = None
    if dist.world == 1 and args.serve_jobs > 0:
        serving = serving_run(args.serve_jobs)

    peak, peak_kind = measured_hbm_peak()
    adjacent = None
    if dist.world == 1 and not args.no_adjacent:
        adjacent = adjacent_rows_run(wl, peak, cpu=not args.no_cpu_baseline)
    step_ms = float(tot.value) / max(int(cnt.value), 1)
    achieved = float(byt.value) / (float(tot.value) * 1e-3) / 1e9 if tot.value > 0 else 0.0
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cs = cpu_sample(args.config, args.cpu_sample_steps)
        cpu = {"value": 1.0 / cs["per_shot_s"], "unit": "shots/s", "cores": 1, "kind": "port",
               "sample": (f"one shot, {cs['nt_sample']} of {cs['nt']} steps of the NumPy oracle migrate "
                          f"({cs['sample_s']:.1f} s), extrapolated linearly in steps and x{cs['migrates_per_shot']} "
                          f"for one migrate per imaging mode as the reference runs them")}
    line = {
        "metric": METRIC, "value": value, "unit": "shots/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded layered model with cavities and a fault; records from the GPU forward model",
        "config": job_config(wl, args, dist.world),
        "gcell_updates_per_s": cell_updates / (total_ms / 1e3) / 1e9,
        "plain": {"value": plain_value, "unit": "shots/s", "ms_per_step": plain_ms / args.steps,
                  "gcell_updates_per_s": cell_updates / (plain_ms / 1e3) / 1e9,
                  "path": "one shot at a time, PP and PS from one pass"},
        "batched_over_plain": value / plain_value,
        "batched_equals_plain": same,
        "e2e": {"value": e2e_value, "unit": "shots/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (None if committed_traffic(f"{wl.engine}_step") is None else
                                 committed_traffic(f"{wl.engine}_step") * float(byt.value) / max(int(cnt.value), 1)),
                     "traffic_note": "DRAM bytes per tick: the ncu-measured DRAM/algorithmic ratio of a captured "
                                     "16-step tick (profiles/) times this run's algorithmic bytes per tick",
                     "kernel": f"{wl.engine} velocity + stress launches of a batched tick (imaging epilogue fused)",
                     "bytes_definition": "per propagator step: Npad*(8*n_state + 4*n_coef) + 8*CPML strip cells*terms;"
                                         " per fused imaging epilogue: 16 B per accumulator, 4 B per replayed field",
                     "bytes_per_tick": float(byt.value) / max(int(cnt.value), 1), "tick_us": step_ms * 1e3,
                     "timed_ticks": int(cnt.value), "peak_source": peak_kind},
        "cpu_baseline": cpu,
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
    # the reference arm is a CPU run on rank 0 alone: no process group, so the
    # other ranks exit at once instead of waiting for rank 0 in a collective
    dist = Dist(join=args.impl != "reference")
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
