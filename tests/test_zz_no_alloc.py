"""The allocation-free stacking entry point agrees with the allocating one.

ertm_stack_noalloc exists for callers that cannot allocate device memory (a
serving process that owns all device memory through its own pool, a host
framework that owns every allocation, code that must not risk the implicit
synchronisation of cudaMalloc/cudaFree).  It keeps its scratch in static
device arrays that every call shares, so this test calls it twice in a row
with different inputs — the second call must not see the first call's sums —
and compares each result with ertm_stack bit for bit (the same float64
accumulation order).  The images are larger than one scratch chunk so the
chunked path is exercised.  This file is collected last on purpose.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stack(lib, fn, images, normalize, out):
    ptrs = (C.c_void_p * len(images))(*[im.data_ptr() for im in images])
    return getattr(lib, fn)(len(images), images[0].numel(), C.cast(ptrs, C.c_void_p), int(normalize),
                            out.data_ptr(), None)


def test_stack_noalloc_matches_ertm_stack_on_two_calls():
    import torch

    from ertm_b200 import _lib

    lib = _lib.lib()
    rng = np.random.default_rng(2024)
    shape = (613, 517)   # 316,921 pixels: more than one 262,144-pixel scratch chunk
    cases = [(5, True, 1.0), (3, True, 7.0), (4, False, 0.3)]
    for n_images, normalize, scale in cases:
        imgs = [torch.from_numpy(rng.normal(scale=scale * (k + 1), size=shape).astype(np.float32)).cuda()
                for k in range(n_images)]
        want = torch.empty(shape, dtype=torch.float32, device="cuda")
        got = torch.full(shape, np.nan, dtype=torch.float32, device="cuda")
        assert _stack(lib, "ertm_stack", imgs, normalize, want) == 0, _lib.last_error()
        assert _stack(lib, "ertm_stack_noalloc", imgs, normalize, got) == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy(), want.cpu().numpy()), (n_images, normalize)


def test_stack_noalloc_rejects_host_pointers_and_too_many_images():
    import torch

    from ertm_b200 import _lib

    lib = _lib.lib()
    dev = [torch.ones(16, device="cuda") for _ in range(2)]
    out = torch.empty(16, device="cuda")
    host = np.ones(16, dtype=np.float32)
    ptrs = (C.c_void_p * 2)(dev[0].data_ptr(), host.ctypes.data)
    assert lib.ertm_stack_noalloc(2, 16, C.cast(ptrs, C.c_void_p), 1, out.data_ptr(), None) != 0
    assert "device memory" in _lib.last_error()
    many = (C.c_void_p * 1025)(*([dev[0].data_ptr()] * 1025))
    assert lib.ertm_stack_noalloc(1025, 16, C.cast(many, C.c_void_p), 1, out.data_ptr(), None) != 0
    assert "1024" in _lib.last_error()


def test_stack_noalloc_single_image_is_a_copy():
    """One image: both entry points return it unchanged (pipeline.py:140-141
    returns a lone image as is), on two calls in a row."""
    import torch

    from ertm_b200 import _lib

    lib = _lib.lib()
    rng = np.random.default_rng(7)
    for scale in (1.0, 50.0):
        img = torch.from_numpy(rng.normal(scale=scale, size=(300, 211)).astype(np.float32)).cuda()
        want = torch.empty_like(img)
        got = torch.full_like(img, np.nan)
        assert _stack(lib, "ertm_stack", [img], True, want) == 0, _lib.last_error()
        assert _stack(lib, "ertm_stack_noalloc", [img], True, got) == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy(), img.cpu().numpy())
        assert np.array_equal(want.cpu().numpy(), img.cpu().numpy())


def test_stack_noalloc_nan_image_left_undivided_like_the_reference():
    """An image holding a NaN has max|image| = NaN in the reference
    (np.max propagates it), so `scale > 0` fails and that image is added
    undivided; the other images are still normalised."""
    import torch

    import oracle as orc
    from ertm_b200 import _lib

    lib = _lib.lib()
    rng = np.random.default_rng(11)
    host = [rng.normal(scale=3.0 * (k + 1), size=(130, 97)).astype(np.float32) for k in range(3)]
    host[1][40, 50] = np.nan
    want = orc.stack_images(host, normalize=True)
    imgs = [torch.from_numpy(h).cuda() for h in host]
    for fn in ("ertm_stack", "ertm_stack_noalloc", "ertm_stack_noalloc"):
        got = torch.empty((130, 97), dtype=torch.float32, device="cuda")
        assert _stack(lib, fn, imgs, True, got) == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy(), want, equal_nan=True), fn
