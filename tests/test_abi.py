"""The C-ABI library loads on any host and exports every declared entry point;
without a GPU, context creation fails with a status, never a crash."""
import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    from tom_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libtomgpu.so not built")
    return _lib


def test_exports_every_declared_symbol():
    L = _lib()
    names = L.declared_symbols()
    assert len(names) >= 25
    raw = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in names if not hasattr(raw, n)]
    assert not missing, missing


def test_status_strings_and_version():
    L = _lib()
    lib = L.lib()
    assert lib.tomgpu_version().startswith(b"tomgpu")
    for s in range(8):
        assert lib.tomgpu_status_string(s)
    assert lib.tomgpu_status_string(99) == b"unknown status"


def test_null_arguments_rejected_without_device():
    L = _lib()
    lib = L.lib()
    assert lib.tomgpu_ctx_create(0, None) == L.TOMGPU_ERR_ARG
    assert lib.tomgpu_rotate3d(None, None, None, None, None, 1, None) == L.TOMGPU_ERR_ARG
    assert lib.tomgpu_match_run_dev(None, None, 0, 0, None, None) == L.TOMGPU_ERR_ARG
    m = (ctypes.c_float * 9)()
    e = (ctypes.c_float * 3)(0, 0, 0)
    assert lib.tomgpu_euler_matrix(e, m) == 0 and list(m) == [1, 0, 0, 0, 1, 0, 0, 0, 1]


def test_context_creation_reports_missing_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib()
    h = ctypes.c_void_p()
    st = L.lib().tomgpu_ctx_create(0, ctypes.byref(h))
    assert st == L.TOMGPU_ERR_CUDA and not h.value
    assert b"device" in L.lib().tomgpu_last_error(None)


def test_host_matrix_equals_oracle(oracle):
    """tomgpu_euler_matrix (host C++) equals the oracle's restatement bit for bit."""
    import numpy as np
    import tom_b200
    rng = np.random.default_rng(5)
    for _ in range(200):
        e = rng.choice([0, 30, 45, 60, 90, 135, 270, 330, 12.5, 77.0, 181.25], 3)
        if rng.random() < 0.5:
            e = (rng.random(3) * 360).astype(np.float32)
        assert np.array_equal(tom_b200.euler_matrix(e), oracle.euler_matrix(e))
