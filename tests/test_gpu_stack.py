"""Per-shot-normalised stacking (pipeline.py:133-161) on the device against
the oracle, bit for bit: host and device images, the split float64 form
(partial sums, then the mean) and stacks larger than one upload group."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


def _images(n_images: int, shape, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_images):
        im = rng.standard_normal(shape).astype(np.float32) * np.float32(10.0 ** rng.uniform(-3, 3))
        if k % 5 == 3:
            im[:] = 0.0                       # an all-zero image is added undivided
        out.append(im)
    return out


def _ptrs(arrs):
    from ertm_b200 import _lib
    return (C.c_void_p * len(arrs))(*[_lib.ptr(a) for a in arrs])


@pytest.mark.parametrize("normalize", [True, False])
def test_stack_of_64_host_and_device_images_equals_oracle(normalize):
    import torch

    from ertm_b200 import _lib
    L = _lib.lib()
    ims = _images(64, (301, 517), 11)
    want = orc.stack_images(ims, normalize=normalize)
    out = np.empty_like(ims[0])
    _lib.check(L.ertm_stack(len(ims), ims[0].size, C.cast(_ptrs(ims), C.c_void_p), int(normalize), _lib.ptr(out),
                            None), "stack")
    assert np.array_equal(out, want)
    # device images, some host images mixed in, device output
    dev = [torch.from_numpy(im).cuda() if k % 3 else im for k, im in enumerate(ims)]
    dout = torch.empty(ims[0].shape, dtype=torch.float32, device="cuda")
    _lib.check(L.ertm_stack(len(dev), ims[0].size, C.cast(_ptrs(dev), C.c_void_p), int(normalize), _lib.ptr(dout),
                            None), "stack")
    assert np.array_equal(dout.cpu().numpy(), want)


def test_partial_sums_in_three_calls_then_finish_equal_oracle():
    import torch

    from ertm_b200 import _lib
    L = _lib.lib()
    ims = _images(23, (97, 211), 5)
    want = orc.stack_images(ims, normalize=True)
    dev = [torch.from_numpy(im).cuda() for im in ims]
    n = ims[0].size
    total = torch.zeros(n, dtype=torch.float64, device="cuda")
    for a, b in ((0, 7), (7, 8), (8, 23)):      # the running sum carries over, image order kept
        part = dev[a:b]
        _lib.check(L.ertm_stack_partial(len(part), n, C.cast(_ptrs(part), C.c_void_p), 1, _lib.ptr(total), None),
                   "partial")
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    _lib.check(L.ertm_stack_finish(n, _lib.ptr(total), len(ims), _lib.ptr(out), None), "finish")
    assert np.array_equal(out.cpu().numpy().reshape(ims[0].shape), want)


def test_stack_larger_than_one_upload_group():
    """Nine host images of 2^25 values (1.2 GB) are staged in two groups;
    the float64 sum carries across them."""
    from ertm_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(2)
    n = 1 << 25
    ims = [(rng.standard_normal(n, dtype=np.float32) * np.float32(k + 1)) for k in range(9)]
    want = orc.stack_images(ims, normalize=True)
    out = np.empty(n, dtype=np.float32)
    _lib.check(L.ertm_stack(len(ims), n, C.cast(_ptrs(ims), C.c_void_p), 1, _lib.ptr(out), None), "stack")
    assert np.array_equal(out, want)


def test_nan_image_left_undivided_in_a_batched_stack():
    from ertm_b200 import _lib
    L = _lib.lib()
    ims = _images(6, (40, 50), 9)
    ims[2] = ims[2].copy()
    ims[2][3, 4] = np.nan
    want = orc.stack_images(ims, normalize=True)
    out = np.empty_like(ims[0])
    _lib.check(L.ertm_stack(len(ims), ims[0].size, C.cast(_ptrs(ims), C.c_void_p), 1, _lib.ptr(out), None), "stack")
    assert np.array_equal(out, want, equal_nan=True)
