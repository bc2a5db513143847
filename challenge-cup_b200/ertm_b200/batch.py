"""Batched migration (form b): many shots per device call.

``BatchMigrator.migrate_shots`` runs a list of shots — possibly on different
models, grids, engines and lengths — through ``ertm_migrate_batch``: all
shots advance together in ticks that share one velocity and one stress
launch per (engine, order) group, and inside each shot the replay of block
b−1 overlaps the backward pass over block b.  Every propagator performs the
same steps in the same order as the plain one-shot path, so each image equals
the plain path's image bit for bit.

Shots are grouped so that a group's device memory (two propagators, the
checkpoints, two replay buffers and the accumulators per shot) stays within a
budget; groups run one after another.  A ``BatchMigrator`` keeps the
propagator pairs it built for the models of its last call and resets them for
the next group or call, so a stream of calls on one model builds the material
tables, CPML profiles and device fields once.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Sequence

import numpy as np

from . import _lib
from .exceptions import ImagingError
from .imaging import MigratorPool, RTMImager, ShotMigrator, pair_device_bytes
from .types import ImageResult


@dataclass
class _Prepared:
    mig: ShotMigrator
    shot: Any
    pairs: list
    store: Any
    start_step: int
    cfg: _lib.MigrateConfig
    record: list[np.ndarray]                     # per component, (nt, nrec) float32
    wavelet: np.ndarray
    modes: tuple[str, ...]
    acc: Any = None


def shot_device_bytes(mig: ShotMigrator, n_steps: int, n_images: int, n_buffers: int = 2,
                      modes: tuple[str, ...] | None = None) -> int:
    """Device memory one shot of a batch holds while it runs: two
    propagators, the checkpoints, the replay buffers (one stored source field
    per step and imaged source wave: P for pp/ps, S for sp/ss), the imaging
    accumulators, and the complex work arrays of the compensated
    viscoacoustic low-pass."""
    info = mig.prop.info()
    state = int(info.state_bytes)
    g = mig.model.grid
    npix = g.nx * g.nz
    interval = max(1, mig.interval_for(n_steps))
    n_states = (n_steps + interval - 1) // interval
    n_src = 2 if modes is None else max(1, len({str(m).lower()[0] for m in modes}))
    replay = n_buffers * interval * n_src * npix * 4
    acc = (2 * n_images + 2) * npix * 8
    lowpass = 0
    q = getattr(mig.back, "q_options", None)
    if mig.engine == "viscoacoustic" and q is not None and q.compensation:
        lowpass = 2 * 16 * info.nzp * info.nxp
    return pair_device_bytes(mig) + n_states * state + replay + acc + lowpass


class BatchMigrator:
    """Migrate many shots per device call with the same imaging settings."""

    def __init__(self, imager: RTMImager, *, memory_budget: int | None = None) -> None:
        self.imager = imager
        self.memory_budget = memory_budget
        # per shot of the last migrate_shots call: its post-processed images,
        # (n_modes, nz, nx) float32 on the device (the host images are copies)
        self.device_images: list = []
        # propagator pairs of the last call's models, reused by the next
        self._pool = MigratorPool(imager)

    def _budget(self) -> int:
        if self.memory_budget is not None:
            return int(self.memory_budget)
        import torch
        free, _ = torch.cuda.mem_get_info()
        # pooled pairs are reused, so the memory they hold is available to
        # the group that takes them
        return int(0.8 * (free + self._pool.held_bytes()))

    def release(self) -> None:
        """Drop the pooled propagator pairs (their device memory is freed)."""
        self._pool.clear()

    def migrate_shots(self, shots: Sequence[Any], models: Any, *, modes: tuple[str, ...] | None = None,
                      wavelets: Sequence[np.ndarray] | None = None) -> list[list[ImageResult]]:
        """Returns, per shot, one ImageResult per mode."""
        modes = tuple(modes or (self.imager.config.mode,))
        model_list = list(models) if isinstance(models, (list, tuple)) else [models] * len(shots)
        if len(model_list) != len(shots):
            raise ImagingError("one model per shot (or one model for all)")
        results: list[list[ImageResult] | None] = [None] * len(shots)
        self.device_images = [None] * len(shots)
        self._pool.begin(model_list)
        checked: set[int] = set()
        for shot, model in zip(shots, model_list):
            try:
                shot.validate()
                if id(model) not in checked:        # one model often serves every shot
                    model.validate()
                    checked.add(id(model))
            except ValueError as exc:
                raise ImagingError(f"invalid imaging input: {exc}") from exc
        group: list[tuple[int, _Prepared]] = []
        taken: dict[int, int] = {}
        used = 0
        budget = self._budget()
        for k, (shot, model) in enumerate(zip(shots, model_list)):
            w = None if wavelets is None else wavelets[k]
            sizer = self._pool.sizer(model)
            need = shot_device_bytes(sizer, sizer.spec.nt if w is None else len(w), len(modes), modes=modes)
            if group and used + need > budget:
                self._run(group, results)
                group, used, taken = [], 0, {}
            mig = self._pool.take(model, taken)
            group.append((k, self._prepare(mig, shot, modes, w)))
            used += need
        if group:
            self._run(group, results)
        return [r for r in results]  # type: ignore[misc]

    def _prepare(self, mig: ShotMigrator, shot: Any, modes, wavelet) -> _Prepared:
        im = self.imager
        record = im._prepare_record(shot, mig.spec, None)
        if not record:
            raise ImagingError("empty shot record; nothing to back-propagate")
        w = im._prepare_wavelet(shot, mig.spec, wavelet)
        pairs, store, start = mig._prepare(shot.source, shot.receivers, modes, len(w))
        names = list(record)
        cfg = mig._config(pairs, names, store, start, len(w))
        rec = [np.ascontiguousarray(record[n], dtype=np.float32) for n in names]
        return _Prepared(mig, shot, pairs, store, start, cfg, rec, w, modes)

    def _run(self, group: list[tuple[int, _Prepared]], results: list) -> None:
        import torch

        shots = (_lib.BatchShot * len(group))()
        keep = []
        for i, (_, p) in enumerate(group):
            g = p.mig.model.grid
            p.acc = torch.zeros((3, len(p.pairs), g.nz, g.nx), dtype=torch.float64, device="cuda")
            rec = torch.empty((len(p.record),) + p.record[0].shape, dtype=torch.float32, device="cuda")
            for c, comp in enumerate(p.record):         # one copy per component, no host-side stacking
                rec[c].copy_(torch.from_numpy(comp))
            keep.append(rec)
            s = shots[i]
            s.fwd = p.mig.prop.handle
            s.back = p.mig.back.handle
            s.cfg = p.cfg
            s.wavelet = _lib.ptr(p.wavelet)
            s.record = _lib.ptr(rec)
            s.num = _lib.ptr(p.acc[0])
            s.illum = _lib.ptr(p.acc[1])
            s.rillum = _lib.ptr(p.acc[2])
        _lib.check(_lib.lib().ertm_migrate_batch(len(group), shots), "migrate_batch")
        L = _lib.lib()
        for k, p in group:
            p.mig.prop._psi_allocated = p.mig.back._psi_allocated = True
            im = self.imager
            cond = str(im.config.condition).lower()
            out = []
            # post-processing reads the accumulators where they are; only the
            # float32 images come back to the host
            g = p.mig.model.grid
            a = p.mig._post_args()
            img = torch.empty((len(p.modes), g.nz, g.nx), dtype=torch.float32, device="cuda")
            for j in range(len(p.modes)):
                _lib.check(L.ertm_postprocess(g.nz, g.nx, float(a["dx"]), float(a["dz"]), _lib.ptr(p.acc[0, j]),
                                              _lib.ptr(p.acc[1, j]), _lib.ptr(p.acc[2, j]), int(a["by_illum"]),
                                              int(a["by_rillum"]), float(a["eps"]), int(bool(a["laplacian"])),
                                              float(a["lowpass_fraction"]), int(a["npml"]),
                                              int(a["boundary"] == "cpml"), _lib.ptr(img[j]), None), "postprocess")
            host = img.cpu().numpy()
            p.acc = None
            self.device_images[k] = img
            for j, m in enumerate(p.modes):
                image = host[j]
                res = ImageResult(image=image, grid=p.mig.model.grid, mode=m,
                                  meta=im._meta(p.mig.spec, p.mig.engine, p.shot, p.store, cond, p.start_step,
                                                p.mig.prop, p.mig.back, m))
                res.meta["batched"] = True
                res.validate()
                out.append(res)
            results[k] = out


@dataclass
class DeviceShot:
    """One shot of a device-resident batched call: its migrator (propagator
    pair, built beforehand and reusable), source, receivers, record
    (contiguous device tensor (n_comp, nt, nrec) at the propagation dt) with
    its component names, wavelet and imaging modes."""
    mig: ShotMigrator
    source: Any
    receivers: Any
    record: Any
    names: Sequence[str]
    wavelet: np.ndarray
    modes: tuple[str, ...] = ("pp",)


def migrate_device_items(items: Sequence[DeviceShot], *, memory_budget: int | None = None):
    """Device-resident batched form over shots that may differ in engine,
    grid, length, components and modes.  Shots run in groups whose device
    footprint fits the budget (default 80 % of free memory); each group is
    one ``ertm_migrate_batch`` call.  Returns, per shot, a device tensor
    (n_modes, nz, nx) float32 of its post-processed images."""
    import torch

    if memory_budget is None:
        free, _ = torch.cuda.mem_get_info()
        memory_budget = int(0.8 * free)
    out: list = [None] * len(items)
    group: list[int] = []
    used = 0
    for k, it in enumerate(items):
        need = shot_device_bytes(it.mig, len(it.wavelet), len(it.modes), modes=tuple(it.modes))
        if group and used + need > memory_budget:
            _run_device_group(items, group, out)
            group, used = [], 0
        group.append(k)
        used += need
    if group:
        _run_device_group(items, group, out)
    return out


def _run_device_group(items: Sequence[DeviceShot], group: list[int], out: list) -> None:
    import torch

    shots = (_lib.BatchShot * len(group))()
    accs = []
    for j, k in enumerate(group):
        it = items[k]
        w = np.ascontiguousarray(it.wavelet, dtype=np.float32)
        pairs, store, start = it.mig._prepare(it.source, it.receivers, tuple(it.modes), len(w))
        cfg = it.mig._config(pairs, list(it.names), store, start, len(w))
        g = it.mig.model.grid
        acc = torch.empty((3, len(pairs), g.nz, g.nx), dtype=torch.float64, device=it.record.device)
        accs.append((acc, w))
        s = shots[j]
        s.fwd, s.back, s.cfg = it.mig.prop.handle, it.mig.back.handle, cfg
        s.wavelet = _lib.ptr(w)
        s.record = _lib.ptr(it.record)
        s.num, s.illum, s.rillum = _lib.ptr(acc[0]), _lib.ptr(acc[1]), _lib.ptr(acc[2])
    _lib.check(_lib.lib().ertm_migrate_batch(len(group), shots), "migrate_batch")
    for j, k in enumerate(group):
        it = items[k]
        mig = it.mig
        mig.prop._psi_allocated = mig.back._psi_allocated = True
        acc = accs[j][0]
        g = mig.model.grid
        imgs = torch.empty((len(it.modes), g.nz, g.nx), dtype=torch.float32, device=acc.device)
        a = mig._post_args()
        for m in range(len(it.modes)):
            _lib.check(_lib.lib().ertm_postprocess(
                g.nz, g.nx, float(a["dx"]), float(a["dz"]), _lib.ptr(acc[0, m]), _lib.ptr(acc[1, m]),
                _lib.ptr(acc[2, m]), int(a["by_illum"]), int(a["by_rillum"]), a["eps"], int(a["laplacian"]),
                a["lowpass_fraction"], int(a["npml"]), int(a["boundary"] == "cpml"), _lib.ptr(imgs[m]), None),
                "postprocess")
        out[k] = imgs


def migrate_device_batch(imager: RTMImager, migrators: Sequence[ShotMigrator], sources: Sequence[Any],
                         receivers: Sequence[Any], records: Sequence[Any], names: Sequence[str],
                         wavelets: Sequence[np.ndarray], *, modes: tuple[str, ...] = ("pp",),
                         memory_budget: int | None = None):
    """Device-resident batched form for shots of one imaging setting: one
    migrator (propagator pair) per shot, built beforehand and reused;
    ``records[k]`` is a contiguous device tensor (n_comp, nt, nrec) aligned
    to the propagation dt.  Returns a list of device tensors (n_modes, nz,
    nx) float32 of final images."""
    del imager   # the migrators carry the imaging settings
    items = [DeviceShot(m, sources[k], receivers[k], records[k], names, wavelets[k], tuple(modes))
             for k, m in enumerate(migrators)]
    return migrate_device_items(items, memory_budget=memory_budget)
