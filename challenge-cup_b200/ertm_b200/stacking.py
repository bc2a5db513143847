"""Per-shot-normalised stacking on the device (pipeline.py:133-161)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .exceptions import PipelineError
from .types import ImageResult


def stack_arrays(images: list[np.ndarray], *, normalize: bool = True) -> np.ndarray:
    """Mean of the images, each divided by its max|·| first when ``normalize``."""
    if not images:
        raise PipelineError("nothing to stack")
    arrs = [np.ascontiguousarray(im, dtype=np.float32) for im in images]
    n = arrs[0].size
    if any(a.size != n for a in arrs):
        raise PipelineError("images differ in size")
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    out = np.empty_like(arrs[0])
    _lib.check(_lib.lib().ertm_stack(len(arrs), n, C.cast(ptrs, C.c_void_p), int(bool(normalize)), _lib.ptr(out),
                                    None), "stack")
    return out


def stack_images(images: list[ImageResult], *, normalize: bool = True) -> ImageResult:
    if not images:
        raise PipelineError("nothing to stack")
    if len(images) == 1:
        return images[0]
    stacked = stack_arrays([im.image for im in images], normalize=normalize)
    meta = dict(images[0].meta)
    meta.update({"stacked": True, "n_shots": len(images), "stack_normalize": bool(normalize)})
    return ImageResult(image=stacked.reshape(images[0].image.shape), grid=images[0].grid, mode=images[0].mode,
                       meta=meta)
