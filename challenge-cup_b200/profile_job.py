"""Profiling tool (not part of the package): one benchmark workload's
migration job, alone in the process, for ncu launch lists and kernel
captures.

    python challenge-cup_b200/profile_job.py \\
        [--config visco] [--nt 48] [--shots 4] [--path batched|plain] [--repeat 2] [--tile-rows 0] [--split 0] [--lanes 0] [--autotune 1] [--lane-assign 0] [--frame-rows 0] [--march 4] [--march-stress 0] [--tma 0] [--save x.npy]

The job is a benchmark step: ``--shots`` shots of the workload migrated
(batched lockstep ticks, or one shot at a time with ``--path plain``) and the
images stacked.  Records come from the GPU forward model first.  Each repeat
is preceded by a 256 MiB fill (the benchmark's L2 flush), which also marks the
start of a repeat in a launch list; the last repeat runs inside the NVTX
range ``job`` (``ncu --nvtx --nvtx-include job/`` captures it alone).  Prints
one JSON line: the launches of this library and the job time per repeat, and
the stencil profiler's per-tick time and bytes over the last repeat.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(prog="python challenge-cup_b200/profile_job.py")
    ap.add_argument("--config", default="visco")
    ap.add_argument("--nt", type=int, default=48)
    ap.add_argument("--shots", type=int, default=None)
    ap.add_argument("--path", choices=("batched", "plain"), default="batched")
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--tile-rows", type=int, default=0, help="stencil tile height 8/16/32 (0: automatic)")
    ap.add_argument("--split", type=int, default=0,
                    help="interior tiles in launches of their own: 0 automatic, 1 never, 2 always")
    ap.add_argument("--lanes", type=int, default=0, help="batched ticks in 1, 2 or 4 stream lanes (0: automatic)")
    ap.add_argument("--autotune", type=int, default=1, help="online autotuning of batched ticks (1 on, 0 off)")
    ap.add_argument("--march", type=int, default=4,
                    help="elastic velocity interiors: 0 tiles, or 2/4/8 chunks per marching segment")
    ap.add_argument("--march-stress", type=int, default=0, help="elastic stress interiors march as well (1)")
    ap.add_argument("--frame-rows", type=int, default=0,
                    help="frame tile height in split launches: 0 the interior's, 8 or 16")
    ap.add_argument("--lane-assign", type=int, default=0,
                    help="two-lane ticks: 0 alternate works (replay | backward), 1 alternate shots")
    ap.add_argument("--tma", type=int, default=0, help="stage interior tiles with TMA (1) or cp.async (0)")
    ap.add_argument("--save", default=None, help="write the stacked images of the last repeat (.npy)")
    ap.add_argument("--lowpass", default=None, metavar="NZxNX",
                    help="time the wavenumber low-pass of one float64 NZxNX array instead of a job")
    ap.add_argument("--line-threads", default="0", metavar="T[,T...]",
                    help="with --lowpass: threads per CTA of the line transforms, one run per value (0: automatic); "
                         "every run's result is compared with the first")
    args = ap.parse_args(argv)

    import torch

    if args.lowpass:
        lowpass_only(args)
        return

    from ertm_b200 import _lib, workloads
    from ertm_b200.batch import migrate_device_batch
    from ertm_b200.imaging import ShotMigrator
    from ertm_b200.propagation import source_wavelet

    L = _lib.lib(0)
    _lib.check(L.ertm_set_tile_rows(args.tile_rows), "tile rows")
    _lib.check(L.ertm_set_tile_split(args.split), "tile split")
    _lib.check(L.ertm_set_tick_lanes(args.lanes), "tick lanes")
    _lib.check(L.ertm_set_autotune(args.autotune), "autotune")
    _lib.check(L.ertm_set_lane_assign(args.lane_assign), "lane assignment")
    _lib.check(L.ertm_set_frame_rows(args.frame_rows), "frame rows")
    _lib.check(L.ertm_set_march(args.march), "march")
    _lib.check(L.ertm_set_march_stress(args.march_stress), "march stress")
    _lib.check(L.ertm_set_tma(args.tma), "tma")
    wl = workloads.WORKLOADS[args.config](seed=0, nt=args.nt)
    if args.shots:
        wl.sources = wl.sources[: args.shots]
    imager, solver = workloads.imager_for(wl)
    shots = workloads.synthesize(wl, solver, wl.sources)
    names = list(wl.components)
    rec = [torch.from_numpy(np.stack([s.components[n] for n in names])).cuda() for s in shots]
    wavelets = [source_wavelet(s, wl.dt, wl.nt) for s in wl.sources]
    g = wl.model.grid
    npix = g.nx * g.nz
    n = len(wl.sources)
    migs = [ShotMigrator(imager, wl.model) for _ in range(n if args.path == "batched" else 1)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    partial = torch.zeros((len(wl.modes), g.nz, g.nx), dtype=torch.float64, device="cuda")
    out = torch.empty((len(wl.modes), g.nz, g.nx), dtype=torch.float32, device="cuda")

    def job():
        if args.path == "batched":
            imgs = migrate_device_batch(imager, migs, wl.sources, [wl.receivers] * n, rec, names, wavelets,
                                        modes=wl.modes)
        else:
            imgs = [migs[0].migrate_device(s, wl.receivers, rec[i], names, wavelets[i], modes=wl.modes)
                    for i, s in enumerate(wl.sources)]
        partial.zero_()
        for k in range(len(wl.modes)):
            ptrs = (C.c_void_p * n)(*[im[k].data_ptr() for im in imgs])
            _lib.check(L.ertm_stack_partial(n, npix, C.cast(ptrs, C.c_void_p), int(n > 1), partial[k].data_ptr(),
                                            None), "stack partial")
            _lib.check(L.ertm_stack_finish(npix, partial[k].data_ptr(), n, out[k].data_ptr(), None), "stack finish")

    launches, job_ms = [], []
    for r in range(args.repeat):
        torch.cuda.synchronize()
        if r == args.repeat - 1:
            _lib.check(L.ertm_profile_stencil(1, 1), "profile")     # the last repeat's ticks
        flush.fill_(1.0)
        before = L.ertm_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        last = r == args.repeat - 1
        if last:
            torch.cuda.nvtx.range_push("job")
        e0.record()
        job()
        e1.record()
        torch.cuda.synchronize()
        if last:
            torch.cuda.nvtx.range_pop()
        job_ms.append(e0.elapsed_time(e1))
        launches.append(int(L.ertm_launch_count() - before))
    if args.save:
        np.save(args.save, out.cpu().numpy())
    tot, cnt, byt = C.c_double(), C.c_int64(), C.c_double()
    _lib.check(L.ertm_profile_read(C.byref(tot), C.byref(cnt), C.byref(byt)), "profile read")
    _lib.check(L.ertm_profile_stencil(0, 1), "profile off")
    ticks = max(int(cnt.value), 1)
    print(json.dumps({"workload": wl.name, "path": args.path, "nt": wl.nt, "shots": n, "launches_per_repeat": launches,
                      "job_ms": job_ms,
                      "stencil_us_per_tick": tot.value / ticks * 1e3, "bytes_per_tick": byt.value / ticks,
                      "timed_ticks": int(cnt.value),
                      "achieved_gbs": byt.value / (tot.value * 1e-3) / 1e9 if tot.value > 0 else None,
                      "checksum": float(out.double().abs().sum().item()),
                      "stage_timeouts": int(L.ertm_stage_timeouts()),
                      "autotune": L.ertm_autotune_report().decode().strip().splitlines()}), flush=True)


def lowpass_only(args) -> None:
    """Repeated ertm_lowpass_wavenumber calls on a device array for each
    --line-threads value (the last repeat of each inside the NVTX range
    ``job``); prints the time per call and whether the result equals the
    first value's."""
    import torch

    from ertm_b200 import _lib
    L = _lib.lib(0)
    nz, nx = (int(v) for v in args.lowpass.lower().split("x"))
    a = torch.randn(nz, nx, dtype=torch.float64, device="cuda")
    b = torch.empty_like(a)
    first = None
    try:
        for threads in (int(v) for v in args.line_threads.split(",")):
            _lib.check(L.ertm_set_line_threads(threads), "line threads")
            ms = []
            for r in range(args.repeat):
                last = r == args.repeat - 1
                torch.cuda.synchronize()
                if last:
                    torch.cuda.nvtx.range_push("job")
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                _lib.check(L.ertm_lowpass_wavenumber(nz, nx, 5.0, 5.0, 0.5, a.data_ptr(), b.data_ptr(), None),
                           "lowpass")
                e1.record()
                torch.cuda.synchronize()
                if last:
                    torch.cuda.nvtx.range_pop()
                ms.append(e0.elapsed_time(e1))
            if first is None:
                first = b.clone()
            print(json.dumps({"lowpass": [nz, nx], "line_threads": threads, "ms_per_call": ms,
                              "equal_to_first": bool(torch.equal(first, b))}), flush=True)
    finally:
        _lib.check(L.ertm_set_line_threads(0), "line threads")


if __name__ == "__main__":
    main()
