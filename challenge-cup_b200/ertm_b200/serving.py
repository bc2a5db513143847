"""Serving loop for migration jobs (continuous batching on one GPU).

A job is the reference pipeline's unit of work: the shots of one model, each
migrated by ``RTMImager.migrate`` (imaging.py:205-349), then stacked per mode
by ``stack_images`` (pipeline.py:133-161).  ``RTMServer`` runs jobs of mixed
engine, grid and length on one device:

* a host thread owns a batch session (``ertm_session_*``): every admitted shot
  advances in the session's lockstep ticks, shots that arrive while others run
  join between ticks, and finished shots leave, so work of different jobs
  overlaps on the device;
* shots are admitted in arrival order while their device footprint (two
  propagators, checkpoints, replay buffers, accumulators, record) fits the
  memory budget (170 GB by default, capped at 90 % of the free memory) and a
  slot is free; checkpoints, wavefields, accumulators and per-shot images stay
  in device memory until the job's stacked images are returned;
* per-shot images are post-processed and stacked on the device
  (``ertm_postprocess``, ``ertm_stack_partial``/``ertm_stack_finish``), and the
  job's future receives host images.

A shot's image does not depend on what else runs in the session: each
propagator performs the same steps in the same order as the one-shot path.
A job whose shot fails to prepare (bad input, a mode the engine cannot image)
fails alone; its shots already on the device run out and are dropped.  So
does a job one of whose shots writes NaN or infinity into a wavefield on the
device (an overflowing or unstable run): the session takes that shot out at
the next poll and the job's future raises NonFiniteWavefieldError.
"""

from __future__ import annotations

import collections
import ctypes as C
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np

from . import _lib
from .exceptions import ImagingError, NonFiniteWavefieldError
from .imaging import RTMImager, ShotMigrator
from .types import ImageResult

DEFAULT_BUDGET = 170 * 10**9


@dataclass
class ServeJob:
    """One migration job: shots on one model, imaged in ``modes`` and stacked."""
    shots: list
    model: Any
    imager: RTMImager
    modes: tuple[str, ...] | None = None
    wavelets: list | None = None
    stack: bool = True
    name: str = ""


@dataclass
class JobResult:
    job_id: int
    name: str
    images: list[ImageResult]                 # stacked per mode (per shot when stack=False: shot-major)
    submitted: float
    finished: float
    shot_finished: list[float] = field(default_factory=list)

    @property
    def latency(self) -> float:
        return self.finished - self.submitted

    @property
    def shot_latencies(self) -> list[float]:
        return [t - self.submitted for t in self.shot_finished]


def shot_footprint_bound(model: Any, imager: RTMImager, n_steps: int, n_modes: int, n_comp: int,
                         nrec: int) -> int:
    """Upper bound of one shot's device bytes, from the grid alone.

    Padded grid (nz+10)·ld with ld = nx+10 rounded up to 32; per propagator
    every field, ψ term and coefficient taken at full padded size; checkpoints
    at the reference's interval (fields-only state bytes, imaging.py:121-124)
    times the full state; two replay buffers of interval·2·nz·nx floats; the
    float64 accumulators; the record and the wavelet; for a compensated
    viscoacoustic backward pass, the two complex work arrays of its
    wavenumber low-pass."""
    from .imaging import checkpoint_interval
    g = model.grid
    engine = imager.solver_config.engine
    L = int(imager.q_config.n_mechanisms) if engine == "viscoacoustic" else 0
    n_fields = {"acoustic": 3, "elastic": 5}.get(engine, 4 + L)
    n_psi = 8 if engine == "elastic" else 4
    nzp, nxp = g.nz + 10, g.nx + 10
    ld = (nxp + 31) // 32 * 32
    fe = nzp * ld
    state = (n_fields + n_psi) * fe * 4
    prop = state + 12 * fe * 4          # coefficient block, Q index and profiles: at most 12 arrays
    field_bytes = n_fields * nzp * nxp * 4
    iv = checkpoint_interval(n_steps, field_bytes, float(imager.config.checkpoint_mb))
    n_states = (n_steps + iv - 1) // iv
    npix = g.nz * g.nx
    replay = 2 * iv * 2 * npix * 4
    acc = (2 * n_modes + 2) * npix * 8 + 3 * n_modes * npix * 8 + n_modes * npix * 4
    record = n_comp * n_steps * nrec * 4 + n_steps * 4
    q = imager.q_config
    lowpass = 2 * 16 * nzp * nxp if engine == "viscoacoustic" and q is not None and q.enabled else 0
    return int(2 * prop + n_states * state + replay + acc + record + lowpass)


def percentile(values, q: float) -> float | None:
    return float(np.percentile(np.asarray(values, dtype=np.float64), q)) if len(values) else None


class _Job:
    def __init__(self, job_id: int, job: ServeJob, future: Future) -> None:
        self.id = job_id
        self.job = job
        self.future = future
        self.modes = tuple(job.modes or (job.imager.config.mode,))
        self.submitted = time.perf_counter()
        self.pending = collections.deque(range(len(job.shots)))
        self.active = 0
        self.images: dict[int, Any] = {}           # shot index -> device tensor (n_modes, nz, nx)
        self.shot_finished: dict[int, float] = {}
        self.free: list[ShotMigrator] = []          # propagator pairs of finished shots, reused
        self.failed: BaseException | None = None
        self.bound: int | None = None


class _Slot:
    def __init__(self, job: _Job, index: int, mig: ShotMigrator, acc, bytes_: int, keep: list) -> None:
        self.job = job
        self.index = index
        self.mig = mig
        self.acc = acc
        self.bytes = bytes_
        self.keep = keep


class RTMServer:
    """Request loop: ``submit`` jobs from any thread, read ``Future`` results."""

    def __init__(self, *, device: int = 0, memory_budget: int | None = None, max_shots: int = 64,
                 ticks_per_poll: int = 64, fault_hook: Callable[[str, int, int], None] | None = None) -> None:
        self.device = int(device)
        self.max_shots = int(max_shots)
        self.ticks_per_poll = int(ticks_per_poll)
        self._budget_request = memory_budget
        self._fault_hook = fault_hook
        self._cv = threading.Condition()
        self._queue: collections.deque[_Job] = collections.deque()
        self._next_id = 0
        self._stop = False
        self._thread: threading.Thread | None = None
        self._error: BaseException | None = None
        self.stats: dict[str, Any] = {"jobs_done": 0, "jobs_failed": 0, "shots_done": 0, "peak_bytes": 0,
                                      "peak_active": 0, "ticks": 0}
        self.shot_latencies: list[float] = []
        self.job_latencies: list[float] = []
        self._prefit_jobs: queue.Queue = queue.Queue()
        self._prefit_thread: threading.Thread | None = None

    # ------------------------------------------------------------------ API
    def start(self) -> "RTMServer":
        if self._thread is None:
            self._stop = False
            self._thread = threading.Thread(target=self._run, name="ertm-serve", daemon=True)
            self._thread.start()
            self._prefit_thread = threading.Thread(target=self._prefit_loop, name="ertm-prefit", daemon=True)
            self._prefit_thread.start()
        return self

    def submit(self, job: ServeJob) -> Future:
        fut: Future = Future()
        with self._cv:
            if self._error is not None:
                raise RuntimeError("the serving loop has stopped") from self._error
            js = _Job(self._next_id, job, fut)
            self._next_id += 1
            self._queue.append(js)
            self._cv.notify()
        solver = getattr(job.imager, "solver_config", None)
        if str(getattr(solver, "engine", "")) == "viscoacoustic":
            self._prefit_jobs.put(job)
        return fut

    def stop(self, timeout: float | None = None) -> None:
        """Finish every submitted job, then end the loop."""
        with self._cv:
            self._stop = True
            self._cv.notify()
        if self._thread is not None:
            self._thread.join(timeout)
            self._thread = None
        if self._prefit_thread is not None:
            self._prefit_jobs.put(None)
            self._prefit_thread.join(timeout)
            self._prefit_thread = None

    def __enter__(self) -> "RTMServer":
        return self.start()

    def __exit__(self, *exc) -> None:
        self.stop()

    def summary(self) -> dict:
        s = dict(self.stats)
        s.update({"shot_latency_p50_s": percentile(self.shot_latencies, 50),
                  "shot_latency_p99_s": percentile(self.shot_latencies, 99),
                  "job_latency_p50_s": percentile(self.job_latencies, 50),
                  "job_latency_p99_s": percentile(self.job_latencies, 99)})
        return s

    # ------------------------------------------------------------- the loop
    def _prefit_loop(self) -> None:
        """Host-only work ahead of admission: the GSLS fits of queued
        viscoacoustic jobs (memoised), done while the device runs other
        shots, so that building their propagators later finds them ready."""
        from .viscoelastic import prefit
        while True:
            job = self._prefit_jobs.get()
            if job is None:
                return
            try:
                q = job.imager.q_config
                prefit(job.model.qp, float(q.f_ref), int(q.n_mechanisms), float(q.band_ratio))
            except Exception:       # the serving loop reports any error when it builds the shot
                pass

    def _run(self) -> None:
        handle = C.c_void_p()
        try:
            import torch
            L = _lib.lib(self.device)        # raises without a usable GPU or library
            torch.cuda.set_device(self.device)
            free, _ = torch.cuda.mem_get_info()
            budget = int(0.9 * free)
            if self._budget_request is not None:
                budget = min(budget, int(self._budget_request))
            else:
                budget = min(budget, DEFAULT_BUDGET)
            self.stats["budget_bytes"] = budget
            _lib.check(L.ertm_session_create(C.byref(handle)), "session create")
        except BaseException as exc:
            with self._cv:
                self._error = exc
            self._fail_all(exc)
            return
        slots: dict[int, _Slot] = {}
        used = 0
        next_tag = 0
        done = (C.c_int64 * 64)()
        n_done = C.c_int32()
        failed = (C.c_int64 * 64)()
        n_failed = C.c_int32()
        t_start = None
        try:
            while True:
                with self._cv:
                    while not self._queue and not slots and not self._stop:
                        self._cv.wait()
                    if self._stop and not self._queue and not slots:
                        break
                # admit shots in arrival order while slots and memory last
                while self._queue and len(slots) < self.max_shots:
                    js = self._queue[0]
                    if js.failed is not None or not js.pending:
                        with self._cv:
                            self._queue.popleft()
                        self._maybe_finish(js)
                        continue
                    i = js.pending[0]
                    try:
                        need = self._bound(js, i)
                    except Exception as exc:
                        self._job_failed(js, exc)
                        continue
                    if used + need > budget:
                        if not slots:
                            self._job_failed(js, ImagingError(
                                f"shot needs ~{need / 1e9:.2f} GB, more than the {budget / 1e9:.2f} GB budget"))
                            continue
                        break
                    try:
                        slot = self._prepare(L, handle, js, i, next_tag, need)
                    except Exception as exc:
                        self._job_failed(js, exc)
                        continue
                    js.pending.popleft()
                    js.active += 1
                    slots[next_tag] = slot
                    next_tag += 1
                    used += slot.bytes
                    if t_start is None:
                        t_start = time.perf_counter()
                    self.stats["peak_bytes"] = max(self.stats["peak_bytes"], used)
                    self.stats["peak_active"] = max(self.stats["peak_active"], len(slots))
                if not slots:
                    continue
                _lib.check(L.ertm_session_advance(handle, self.ticks_per_poll, done, len(done), C.byref(n_done)),
                           "session advance")
                # shots whose wavefields became non-finite left the session: their jobs fail, others run on
                while True:
                    _lib.check(L.ertm_session_take_failed(handle, failed, len(failed), C.byref(n_failed)),
                               "session failed shots")
                    for k in range(n_failed.value):
                        slot = slots.pop(int(failed[k]))
                        used -= slot.bytes
                        self._shot_failed(slot)
                    if n_failed.value < len(failed):
                        break
                for k in range(n_done.value):
                    slot = slots.pop(int(done[k]))
                    used -= slot.bytes
                    self._shot_done(L, slot)
            self.stats["ticks"] = int(L.ertm_session_ticks(handle))
            if t_start is not None:
                self.stats["busy_s"] = time.perf_counter() - t_start
        except BaseException as exc:          # device or library failure: every job still open fails
            with self._cv:
                self._error = exc
            self._fail_all(exc, slots)
        finally:
            L.ertm_session_destroy(handle)

    # ------------------------------------------------------------- helpers
    def _bound(self, js: _Job, i: int) -> int:
        if js.bound is None:
            job = js.job
            shot = job.shots[i]
            comps = dict(getattr(shot, "components", {}) or {}) or {"primary": shot.data}
            nrec = int(np.asarray(shot.data).shape[1]) if np.ndim(shot.data) == 2 else 0
            spec_nt = int(job.imager.solver_config.nt)
            js.bound = shot_footprint_bound(job.model, job.imager, spec_nt, len(js.modes), len(comps), nrec)
        return js.bound

    def _prepare(self, L, handle, js: _Job, i: int, tag: int, need: int) -> _Slot:
        import torch
        if self._fault_hook is not None:
            self._fault_hook("prepare", js.id, i)
        job = js.job
        mig = js.free.pop() if js.free else ShotMigrator(job.imager, job.model)
        shot = job.shots[i]
        im = job.imager
        if hasattr(shot, "validate"):
            try:
                shot.validate()
            except ValueError as exc:
                raise ImagingError(f"invalid imaging input: {exc}") from exc
        record = im._prepare_record(shot, mig.spec, None)
        if not record:
            raise ImagingError("empty shot record; nothing to back-propagate")
        w = im._prepare_wavelet(shot, mig.spec, None if job.wavelets is None else job.wavelets[i])
        pairs, store, start = mig._prepare(shot.source, shot.receivers, js.modes, len(w))
        names = list(record)
        cfg = mig._config(pairs, names, store, start, len(w))
        rec = np.ascontiguousarray(np.stack([np.asarray(record[n], dtype=np.float32) for n in names]))
        g = mig.model.grid
        acc = torch.zeros((3, len(pairs), g.nz, g.nx), dtype=torch.float64, device="cuda")
        s = _lib.BatchShot()
        s.fwd, s.back, s.cfg = mig.prop.handle, mig.back.handle, cfg
        s.wavelet = _lib.ptr(w)
        s.record = _lib.ptr(rec)
        s.num, s.illum, s.rillum = _lib.ptr(acc[0]), _lib.ptr(acc[1]), _lib.ptr(acc[2])
        _lib.check(L.ertm_session_add(handle, C.byref(s), tag), "session add")
        return _Slot(js, i, mig, acc, need, [w])

    def _shot_done(self, L, slot: _Slot) -> None:
        import torch
        js = slot.job
        js.active -= 1
        mig = slot.mig
        mig.prop._psi_allocated = mig.back._psi_allocated = True
        now = time.perf_counter()
        js.shot_finished[slot.index] = now
        self.shot_latencies.append(now - js.submitted)
        self.stats["shots_done"] += 1
        if js.failed is None:
            try:
                if self._fault_hook is not None:
                    self._fault_hook("finish", js.id, slot.index)
                g = mig.model.grid
                n_modes = slot.acc.shape[1]
                imgs = torch.empty((n_modes, g.nz, g.nx), dtype=torch.float32, device=slot.acc.device)
                a = mig._post_args()
                for k in range(n_modes):
                    _lib.check(L.ertm_postprocess(
                        g.nz, g.nx, float(a["dx"]), float(a["dz"]), _lib.ptr(slot.acc[0, k]),
                        _lib.ptr(slot.acc[1, k]), _lib.ptr(slot.acc[2, k]), int(a["by_illum"]),
                        int(a["by_rillum"]), a["eps"], int(a["laplacian"]), a["lowpass_fraction"], int(a["npml"]),
                        int(a["boundary"] == "cpml"), _lib.ptr(imgs[k]), None), "postprocess")
                js.images[slot.index] = imgs
            except Exception as exc:
                self._job_failed(js, exc)
        js.free.append(mig)
        self._maybe_finish(js)

    def _shot_failed(self, slot: _Slot) -> None:
        """A shot whose wavefield became non-finite on the device: its job
        fails (once its other running shots have left the session); the
        propagator pair is dropped rather than reused."""
        js = slot.job
        js.active -= 1
        self.stats["shots_failed"] = self.stats.get("shots_failed", 0) + 1
        self._job_failed(js, NonFiniteWavefieldError(
            f"shot {slot.index} of job {js.job.name!r}: a wavefield became non-finite (NaN or infinity) on the "
            f"device"))

    def _maybe_finish(self, js: _Job) -> None:
        if js.active or js.future.done():
            return
        if js.failed is not None:
            js.free.clear()
            js.images.clear()
            self.stats["jobs_failed"] += 1
            js.future.set_exception(js.failed)
            return
        if js.pending:
            return
        try:
            res = self._assemble(js)
        except Exception as exc:
            js.failed = exc
            self.stats["jobs_failed"] += 1
            js.future.set_exception(exc)
            return
        finally:
            js.free.clear()
        js.images.clear()
        self.stats["jobs_done"] += 1
        self.job_latencies.append(res.latency)
        js.future.set_result(res)

    def _assemble(self, js: _Job) -> JobResult:
        import torch
        job = js.job
        n = len(job.shots)
        g = job.model.grid
        npix = g.nz * g.nx
        L = _lib.lib()
        metas = {"job": job.name, "n_shots": n, "served": True}
        out: list[ImageResult] = []
        if job.stack:
            partial = torch.zeros((len(js.modes), g.nz, g.nx), dtype=torch.float64, device="cuda")
            final = torch.empty((len(js.modes), g.nz, g.nx), dtype=torch.float32, device="cuda")
            for k in range(len(js.modes)):
                ptrs = (C.c_void_p * n)(*[js.images[i][k].data_ptr() for i in range(n)])
                _lib.check(L.ertm_stack_partial(n, npix, C.cast(ptrs, C.c_void_p), int(n > 1),
                                                _lib.ptr(partial[k]), None), "stack partial")
                _lib.check(L.ertm_stack_finish(npix, _lib.ptr(partial[k]), n, _lib.ptr(final[k]), None),
                           "stack finish")
            host = final.cpu().numpy()
            for k, m in enumerate(js.modes):
                out.append(ImageResult(image=host[k], grid=g, mode=m,
                                       meta={**metas, "stacked": n > 1, "stack_normalize": n > 1}).validate())
        else:
            for i in range(n):
                host = js.images[i].cpu().numpy()
                for k, m in enumerate(js.modes):
                    out.append(ImageResult(image=host[k], grid=g, mode=m, meta={**metas, "shot": i}).validate())
        return JobResult(job_id=js.id, name=job.name, images=out, submitted=js.submitted,
                         finished=time.perf_counter(), shot_finished=[js.shot_finished[i] for i in range(n)])

    def _job_failed(self, js: _Job, exc: BaseException) -> None:
        if js.failed is None:
            js.failed = exc
        js.pending.clear()
        self._maybe_finish(js)

    def _fail_all(self, exc: BaseException, slots: dict | None = None) -> None:
        jobs = {id(s.job): s.job for s in (slots or {}).values()}
        with self._cv:
            for js in self._queue:
                jobs[id(js)] = js
            self._queue.clear()
        for js in jobs.values():
            if not js.future.done():
                js.future.set_exception(exc)
                self.stats["jobs_failed"] += 1
