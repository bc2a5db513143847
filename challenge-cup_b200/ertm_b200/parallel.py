"""Shot-parallel migration: one process per GPU, shots sharded across ranks.

Shots are independent, so a job partitions into per-rank shards with no
exchange while the wavefields propagate.  Each rank migrates its shard with the
batched path (``BatchMigrator``), then adds its per-shot-normalised images into
a float64 sum on its own GPU (``ertm_stack_partial``).  One all-reduce of that
``(n_modes, nz, nx)`` float64 sum is the job's only collective; every rank then
divides by the job's shot count and casts to float32 (``ertm_stack_finish``).
This is ``stack_images`` (pipeline.py:133-161) with its accumulation loop split
across GPUs: the float64 sum keeps the result within float64 rounding of the
one-process stack.

Before the sum, the ranks exchange a status flag, so that a rank whose shard
failed makes every rank raise ``ShardError`` instead of leaving the others
waiting inside the all-reduce; every rank takes the same collective steps in
the same order on the success and the error path.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, Callable, Sequence

import numpy as np

from . import _lib
from .exceptions import ImagingError
from .types import ImageResult

# algorithmic bytes per padded cell and step (fields read+written, coefficients read)
_BYTES_PER_CELL = {"acoustic": 36.0, "elastic": 60.0, "viscoacoustic": 92.0}


class ShardError(RuntimeError):
    """A rank's shard failed; raised on every rank of the job."""


def shot_cost(nx: int, nz: int, nt: int, engine: str) -> float:
    """Relative work of one shot: cells x steps x bytes per cell-step."""
    return float(nx) * float(nz) * float(nt) * _BYTES_PER_CELL.get(engine, 60.0)


def plan_shards(costs: Sequence[float], world: int) -> list[list[int]]:
    """Largest-first greedy bin packing of shot indices onto ``world`` ranks.

    Shots are taken in order of decreasing cost (ties: lower index first) and
    each goes to the rank with the least load so far (ties: lower rank).  The
    plan depends only on ``costs`` and ``world``, so every rank computes the
    same plan without communicating.  Each rank's list is in shot order."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    loads = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        shards[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(s) for s in shards]


def _collective_device(group) -> str:
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return f"cuda:{torch.cuda.current_device()}"
    return "cpu"


def exchange_status(failed: bool, group=None) -> int:
    """All-reduce of a failure flag: the number of ranks whose shard failed."""
    import torch
    import torch.distributed as dist
    flag = torch.tensor([1 if failed else 0], dtype=torch.int64, device=_collective_device(group))
    dist.all_reduce(flag, op=dist.ReduceOp.SUM, group=group)
    return int(flag.item())


def reduce_partial_sums(partial, group=None):
    """Sum the ranks' float64 partial stacks in place (the one data collective)."""
    import torch.distributed as dist
    dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=group)
    return partial


@dataclass
class ShardResult:
    """What one rank contributes: its float64 partial sums and shot count."""
    partial: Any            # torch float64 tensor (n_modes, nz, nx)
    count: int
    per_shot: list          # per local shot: list of ImageResult (one per mode)


def _device_partial(images_per_mode: Sequence[Sequence[Any]], shape, normalize: bool):
    """float64 partial sums (n_modes, nz, nx) on the current GPU; the images
    are float32 host arrays or contiguous device tensors."""
    import torch
    L = _lib.lib()
    n = int(np.prod(shape))
    out = torch.zeros((len(images_per_mode),) + tuple(shape), dtype=torch.float64, device="cuda")
    for k, imgs in enumerate(images_per_mode):
        arrs = [im if hasattr(im, "data_ptr") else np.ascontiguousarray(im, dtype=np.float32) for im in imgs]
        if not arrs:
            continue
        ptrs = (C.c_void_p * len(arrs))(*[_lib.ptr(a) for a in arrs])
        _lib.check(L.ertm_stack_partial(len(arrs), n, C.cast(ptrs, C.c_void_p), int(bool(normalize)),
                                        _lib.ptr(out[k]), None), "stack partial")
    return out


def _device_finish(total, count: int):
    import torch
    L = _lib.lib()
    out = torch.empty(total.shape, dtype=torch.float32, device=total.device)
    n = int(total[0].numel())
    for k in range(total.shape[0]):
        _lib.check(L.ertm_stack_finish(n, _lib.ptr(total[k]), int(count), _lib.ptr(out[k]), None), "stack finish")
    return out


class ShotParallelMigrator:
    """Migrate and stack one job's shots over all ranks of a process group.

    Every rank calls ``migrate_job`` with the same full list of shots; each
    migrates the shard ``plan_shards`` gives it and all ranks return the same
    stacked images (one ``ImageResult`` per mode)."""

    def __init__(self, imager, *, group=None, memory_budget: int | None = None, normalize: bool = True,
                 local: Callable | None = None, finish: Callable | None = None) -> None:
        self.imager = imager
        self.group = group
        self.memory_budget = memory_budget
        self.normalize = bool(normalize)
        self._local = local or self._migrate_local
        self._finish = finish or _device_finish
        self._batch = None      # one BatchMigrator across jobs: its propagator pairs are reused

    def release(self) -> None:
        """Free the propagator pairs kept from the last job."""
        if self._batch is not None:
            self._batch.release()

    def _migrate_local(self, shots, models, modes, wavelets, normalize: bool) -> ShardResult:
        from .batch import BatchMigrator
        if not shots:
            g = models.grid if not isinstance(models, (list, tuple)) else None
            shape = (g.nz, g.nx) if g is not None else (0, 0)
            import torch
            return ShardResult(torch.zeros((len(modes),) + shape, dtype=torch.float64, device="cuda"), 0, [])
        if self._batch is None:
            self._batch = BatchMigrator(self.imager, memory_budget=self.memory_budget)
        bm = self._batch
        per_shot = bm.migrate_shots(shots, models, modes=modes, wavelets=wavelets)
        shape = per_shot[0][0].image.shape
        # the images are still on the device: stack them there
        partial = _device_partial([[d[k] for d in bm.device_images] for k in range(len(modes))], shape, normalize)
        return ShardResult(partial, len(per_shot), per_shot)

    def migrate_job(self, shots: Sequence[Any], models: Any, *, modes: tuple[str, ...] | None = None,
                    wavelets: Sequence[np.ndarray] | None = None) -> list[ImageResult]:
        import torch.distributed as dist
        modes = tuple(modes or (self.imager.config.mode,))
        world = dist.get_world_size(self.group) if dist.is_initialized() else 1
        rank = dist.get_rank(self.group) if dist.is_initialized() else 0
        model_list = list(models) if isinstance(models, (list, tuple)) else [models] * len(shots)
        if len(model_list) != len(shots):
            raise ImagingError("one model per shot (or one model for all)")
        if not shots:
            raise ImagingError("a job needs at least one shot")
        grids = {(m.grid.nz, m.grid.nx) for m in model_list}
        if len(grids) != 1:
            raise ImagingError("shots stacked into one image must share the model grid")
        costs = [shot_cost(m.grid.nx, m.grid.nz, int(s.data.shape[0]), self.imager.solver_config.engine)
                 for s, m in zip(shots, model_list)]
        mine = plan_shards(costs, world)[rank]
        normalize = self.normalize and len(shots) > 1
        error: BaseException | None = None
        try:
            local = self._local([shots[i] for i in mine], [model_list[i] for i in mine] if mine else model_list[0],
                                modes, None if wavelets is None else [wavelets[i] for i in mine], normalize)
        except Exception as exc:      # reported to every rank below, then re-raised
            error, local = exc, None
        failed = exchange_status(error is not None, self.group) if world > 1 else int(error is not None)
        if failed:
            msg = f"{failed} of {world} rank(s) failed to migrate their shard"
            raise ShardError(msg) from error
        total = reduce_partial_sums(local.partial, self.group) if world > 1 else local.partial
        images = self._finish(total, len(shots))
        host = images.cpu().numpy() if hasattr(images, "cpu") else np.asarray(images)
        g = model_list[0].grid
        out = []
        for k, m in enumerate(modes):
            meta = {"stacked": len(shots) > 1, "n_shots": len(shots), "stack_normalize": normalize,
                    "ranks": world, "shard": list(mine), "mode": m}
            if local.per_shot:
                meta = {**local.per_shot[0][k].meta, **meta}
            res = ImageResult(image=host[k].reshape(g.nz, g.nx), grid=g, mode=m, meta=meta)
            out.append(res)
        return out
