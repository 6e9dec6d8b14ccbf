"""The allocation-free top-K entry point (tomgpu_topk_noalloc_dev) gives the same
peaks as the allocating tomgpu_topk_dev, on two calls in a row.

Callers that cannot allocate device memory when they need peaks (under a
framework that owns the device memory, in loops that may not risk an
allocation failure) use this entry point; its scratch is a fixed 2^24-voxel
device array.  The file name sorts
last so a run that stops at the first failure has already run the rest."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _volume():
    rng = np.random.default_rng(99)
    v = rng.standard_normal((96, 80, 64)).astype(np.float32)
    for p in [(10, 20, 30), (50, 60, 10), (90, 5, 60), (40, 40, 40)]:
        v[p] = 9.0 + p[0] / 100.0
    return v


def test_noalloc_topk_matches_allocating_entry_point(gpu):
    import torch
    from tom_b200 import _lib
    from tom_b200.tom import _cdims, _tptr
    lib = _lib.lib()
    vol = _volume()
    K, radius = 25, 3.0
    dev = gpu.to_device(vol)
    ref_vals, ref_pos = gpu.topk_peaks(dev, K, radius)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        vals = torch.full((K,), float("nan"), dtype=torch.float32, device="cuda")
        pos = torch.full((K, 3), -7, dtype=torch.int32, device="cuda")
        st = lib.tomgpu_topk_noalloc_dev(ctypes.c_void_p(stream), _tptr(dev), _cdims(vol.shape), K, radius,
                                         _tptr(vals), _tptr(pos))
        assert st == 0, lib.tomgpu_last_error(None)
        torch.cuda.synchronize()
        assert np.array_equal(vals.cpu().numpy(), ref_vals), call
        assert np.array_equal(pos.cpu().numpy(), ref_pos), call
    # the input is left untouched
    assert np.array_equal(gpu.from_device(dev), vol)


def test_noalloc_topk_rejects_oversized_volume(gpu):
    import torch
    from tom_b200 import _lib
    from tom_b200.tom import _cdims, _tptr
    lib = _lib.lib()
    small = torch.zeros(8, device="cuda")
    vals = torch.empty(4, device="cuda")
    pos = torch.empty(12, dtype=torch.int32, device="cuda")
    st = lib.tomgpu_topk_noalloc_dev(None, _tptr(small), _cdims((512, 512, 256)), 4, 2.0, _tptr(vals), _tptr(pos))
    assert st == _lib.TOMGPU_ERR_UNSUPPORTED
    assert b"16777216" in lib.tomgpu_last_error(None)
    for bad in (float("inf"), float("nan")):
        st = lib.tomgpu_topk_noalloc_dev(None, _tptr(small), _cdims((2, 2, 2)), 4, bad, _tptr(vals), _tptr(pos))
        assert st == _lib.TOMGPU_ERR_ARG, bad
